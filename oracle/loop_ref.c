/*
 * ORACLE (test infrastructure only) -- C restatement of one time step of
 * StaRMAP's starmap_solver.m (the Strang-split update, lines 307-421).
 *
 * Used only by the test suite, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py, as the checker and as the timed CPU baseline; the product
 * library never links or calls it.  It is written independently of the GPU
 * code: it walks the reference's boundary-extension index vectors
 * (starmap_solver.m:127-132) literally, forms every difference as
 * (U[ext[p+1]] - U[ext[p]]) / h like `diff(U(ext,:,:))/h`, folds the coupling
 * terms in `sumcell` order (starmap_solver.m:516-519) and evaluates the update
 * U + dt/2*(W+Q-s.*U).*E with MATLAB's left-to-right order.  Compiled without
 * FMA contraction (-ffp-contract=off) so that results match the numpy
 * restatement in oracle/solver_np.py bit for bit.  Parallelised with OpenMP
 * over destination rows; sources and destinations of a phase are disjoint.
 */
#include <stdint.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    const double* p; /* column-major array with the component's extents, or NULL */
    double s;        /* scalar value when p == NULL */
} ofield;

typedef struct {
    int32_t n_sys;
    int32_t n[3];
    int32_t bc[3];
    double h[3];
    double hdt;            /* dt/2 */
    int32_t filter_mode;   /* 0 none, 1 substep, 2 full */
    const int32_t* ext;    /* [3*n_sys] extents per component */
    const int32_t* gt;     /* [3*n_sys] grid types (1/2) */
    const int32_t* cptr;   /* [n_sys+1] coupling list offsets (sumcell order) */
    const int32_t* csrc;   /* source component */
    const int32_t* cdir;   /* direction 0,1,2 (Mx, My, Mz) */
    const double* cw;      /* M_d(j,i) */
    const int32_t* destA;  /* outer set c211,c121,c112,c222 */
    int32_t nA;
    const int32_t* destB;  /* inner set c111,c221,c212,c122 */
    int32_t nB;
    const ofield* sT;      /* per component */
    const ofield* ET;
    const ofield* Q;
    const ofield* F1;      /* substep k=1 or full */
    const ofield* F2;      /* substep k=2 */
    ofield sA1, EA;
} oracle_desc;

static inline double fv(const ofield* f, long i) { return f->p ? f->p[i] : f->s; }

/* extension vector of starmap_solver.m:127-132 (0-based), length out+1 */
static int* make_ext(int n, int bc, int g, int* len) {
    int* e;
    int k = 0, i;
    if (g == 1) {
        e = (int*)malloc(sizeof(int) * (n + 2));
        for (i = 0; i < bc; ++i) e[k++] = i;
        for (i = 0; i < n; ++i) e[k++] = i;
        e[k++] = bc * (n - 1);
    } else {
        int n2 = n + bc;
        e = (int*)malloc(sizeof(int) * (n2 + 1));
        for (i = 0; i < 1 - bc; ++i) e[k++] = n2 - 1;
        for (i = 0; i < n2; ++i) e[k++] = i;
    }
    *len = k;
    return e;
}

static inline double upd(double u, double W, double q, double s, double E, double hdt) {
    double t = W + q;
    t = t - s * u;
    t = hdt * t;
    t = t * E;
    return u + t;
}

static void phase(const oracle_desc* d, double* const* U, int* ext_v[3][2], const int32_t* dest, int nd,
                  int is_b, int kf) {
    long rows_total = 0;
    int q;
    long* row_off = (long*)malloc(sizeof(long) * (nd + 1));
    for (q = 0; q < nd; ++q) {
        const int j = dest[q];
        row_off[q] = rows_total;
        rows_total += (long)d->ext[3 * j + 1] * d->ext[3 * j + 2];
    }
    row_off[nd] = rows_total;
    long r;
#pragma omp parallel for schedule(dynamic, 4)
    for (r = 0; r < rows_total; ++r) {
        int lo_q = 0, hi_q = nd - 1;   /* destination owning row r */
        while (lo_q < hi_q) {
            const int mid = (lo_q + hi_q + 1) / 2;
            if (row_off[mid] <= r) lo_q = mid; else hi_q = mid - 1;
        }
        const int qq = lo_q;
        const int j = dest[qq];
        const long rr = r - row_off[qq];
        const int e0 = d->ext[3 * j], e1 = d->ext[3 * j + 1];
        const int i1 = (int)(rr % e1), i2 = (int)(rr / e1);
        double* Uj = U[j];
        int i0;
        for (i0 = 0; i0 < e0; ++i0) {
            const int idx[3] = {i0, i1, i2};
            double S = 0.0;
            int c;
            for (c = d->cptr[j]; c < d->cptr[j + 1]; ++c) {
                const int i = d->csrc[c], dir = d->cdir[c];
                const int g = d->gt[3 * i + dir];
                const int* E = ext_v[dir][g - 1];
                int lo[3] = {idx[0], idx[1], idx[2]}, hi[3] = {idx[0], idx[1], idx[2]};
                lo[dir] = E[idx[dir]];
                hi[dir] = E[idx[dir] + 1];
                const long se0 = d->ext[3 * i], se1 = d->ext[3 * i + 1];
                const double a = U[i][hi[0] + se0 * (hi[1] + se1 * hi[2])];
                const double b = U[i][lo[0] + se0 * (lo[1] + se1 * lo[2])];
                const double du = (a - b) / d->h[dir];
                const double term = du * d->cw[c];
                S = (c == d->cptr[j]) ? term : S + term;
            }
            const double W = -S;
            const long li = i0 + (long)e0 * (i1 + (long)e1 * i2);
            double u = Uj[li];
            const double qv = fv(&d->Q[j], li);
            if (!is_b) {
                u = upd(u, W, qv, fv(&d->sT[j], li), fv(&d->ET[j], li), d->hdt);
                if (d->filter_mode == 1) u = u * fv(kf == 1 ? &d->F1[j] : &d->F2[j], li);
            } else if (j == 0) {
                const double s = fv(&d->sA1, li), Ea = fv(&d->EA, li);
                u = upd(u, W, qv, s, Ea, d->hdt);
                u = upd(u, W, qv, s, Ea, d->hdt);
            } else {
                const double s = fv(&d->sT[j], li), Et = fv(&d->ET[j], li);
                u = upd(u, W, qv, s, Et, d->hdt);
                if (d->filter_mode == 1) u = u * fv(&d->F1[j], li);
                u = upd(u, W, qv, s, Et, d->hdt);
                if (d->filter_mode == 1) u = u * fv(&d->F2[j], li);
            }
            Uj[li] = u;
        }
    }
    free(row_off);
}

/* One step A(k=1) B A(k=2) [full filter]; returns 0. */
int oracle_step(const oracle_desc* d, double* const* U, int nthreads) {
    int* ext_v[3][2];
    int dd, g, len;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    for (dd = 0; dd < 3; ++dd)
        for (g = 1; g <= 2; ++g) ext_v[dd][g - 1] = make_ext(d->n[dd], d->bc[dd], g, &len);
    phase(d, U, ext_v, d->destA, d->nA, 0, 1);
    phase(d, U, ext_v, d->destB, d->nB, 1, 0);
    phase(d, U, ext_v, d->destA, d->nA, 0, 2);
    if (d->filter_mode == 2) {
        int j;
        for (j = 1; j < d->n_sys; ++j) {
            const long m = (long)d->ext[3 * j] * d->ext[3 * j + 1] * d->ext[3 * j + 2];
            long i;
            double* Uj = U[j];
#pragma omp parallel for
            for (i = 0; i < m; ++i) Uj[i] = Uj[i] * fv(&d->F1[j], i);
        }
    }
    for (dd = 0; dd < 3; ++dd)
        for (g = 0; g < 2; ++g) free(ext_v[dd][g]);
    return 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
