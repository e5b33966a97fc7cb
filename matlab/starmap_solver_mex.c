/*
 * starmap_solver_mex.c -- MATLAB / GNU Octave gateway of the B200 time loop.
 *
 * Called by matlab/starmap_solver.m, the drop-in for the reference's
 * output = starmap_solver(par) (starmap_solver.m:1): the .m file does the
 * host setup of starmap_solver.m:55-305 (grid types, staggered grids, hook
 * sampling, first-step materials, dt, decay factors, sources and filter
 * tables) and hands the arrays to this gateway once; the gateway runs the
 * whole update loop of starmap_solver.m:307-421 on the GPU through the C ABI
 * of include/starmap_gpu.h and returns the final components.
 *
 *   [U, ms] = starmap_solver_mex(desc, U0, dt, nsteps)
 *   gt      = starmap_solver_mex('classify', Mx, My, Mz)
 *
 *   desc     struct with the fields of smg_problem, MATLAB-style:
 *              n, bc, h      1x3 (solver ordering; 2D: n = [1 nx ny])
 *              gt            n_sys x 3 grid types (1 or 2)
 *              Mx, My, Mz    n_sys x n_sys full double
 *              fields        1 x nf cell: one double array per coefficient
 *                            field (sT1{g,m}, ET{g,m}, sA1, EA, Q{j},
 *                            filterTerm{g,m[,k]}); one element = a scalar
 *              field_grid    nf x 3 grid type of each field
 *              sigma_t, decay_t, source, filter1, filter2
 *                            1 x n_sys field numbers (1-based; 0 = none)
 *              sigma_a, decay_a   field numbers (1-based)
 *              filter_mode   0 none, 1 'substep', 2 'full'
 *   U0       1 x n_sys cell, component j on its staggered grid
 *   dt       time step;  nsteps  number of full Strang steps
 *   U        1 x n_sys cell, the components after nsteps steps (same sizes)
 *   ms       device time of the loop in milliseconds
 *   gt       n_sys x 3 grid types of the components from the sparsity of
 *            Mx/My/Mz (starmap_solver.m:76-98, smg_classify)
 *
 * Build:  mex -R2018a starmap_solver_mex.c -I../include -L../starmap_b200 -lstarmap_gpu
 *    or:  mkoctfile --mex starmap_solver_mex.c -I../include -L../starmap_b200 -lstarmap_gpu
 * Errors are raised with the identifier starmap:gpu (library failures carry
 * the library's message) and the GPU handle is released first.
 */
#include <stdint.h>
#include <string.h>

#include "mex.h"
#include "starmap_gpu.h"

static const mxArray* desc_field(const mxArray* d, const char* name) {
    const mxArray* f = mxGetField(d, 0, name);
    if (!f) mexErrMsgIdAndTxt("starmap:gpu:desc", "descriptor field '%s' is missing", name);
    return f;
}

/* a real, full double array of `count` elements (count 0: any size) */
static const double* dbl(const mxArray* a, const char* name, size_t count) {
    if (!mxIsDouble(a) || mxIsComplex(a) || mxIsSparse(a))
        mexErrMsgIdAndTxt("starmap:gpu:desc", "'%s' must be a real full double array", name);
    if (count && mxGetNumberOfElements(a) != count)
        mexErrMsgIdAndTxt("starmap:gpu:desc", "'%s' must have %d elements", name, (int)count);
    return mxGetPr(a);
}

/* whole number in [lo, hi] */
static int32_t whole(double v, int lo, int hi, const char* name) {
    if (!(v >= lo && v <= hi) || v != (double)(int32_t)v)
        mexErrMsgIdAndTxt("starmap:gpu:desc", "'%s' must hold whole numbers in %d..%d", name, lo, hi);
    return (int32_t)v;
}

/* 1-based field numbers (0 = none) -> 0-based indices (-1 = none) */
static int32_t* index_table(const mxArray* d, const char* name, int n_sys, int nf) {
    const double* v = dbl(desc_field(d, name), name, (size_t)n_sys);
    int32_t* out = (int32_t*)mxMalloc(sizeof(int32_t) * (size_t)n_sys);
    for (int j = 0; j < n_sys; ++j) out[j] = whole(v[j], 0, nf, name) - 1;
    return out;
}

static void check(int rc, smg_handle* h) {
    if (rc < 0) {
        char msg[1024];
        strncpy(msg, smg_last_error(h), sizeof msg - 1);
        msg[sizeof msg - 1] = '\0';
        if (h) smg_destroy(h);
        mexErrMsgIdAndTxt("starmap:gpu", "starmap GPU library (code %d): %s", rc, msg);
    }
}

/* gt = starmap_solver_mex('classify', Mx, My, Mz) */
static void classify(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    if (nrhs != 4 || nlhs > 1) mexErrMsgIdAndTxt("starmap:gpu:usage", "usage: gt = starmap_solver_mex('classify', Mx, My, Mz)");
    const int n_sys = (int)mxGetM(prhs[3]);
    if (n_sys < 1 || mxGetN(prhs[3]) != (size_t)n_sys) mexErrMsgIdAndTxt("starmap:gpu:desc", "'Mz' must be square");
    const double* Mx = dbl(prhs[1], "Mx", (size_t)n_sys * n_sys);
    const double* My = dbl(prhs[2], "My", (size_t)n_sys * n_sys);
    const double* Mzv = dbl(prhs[3], "Mz", (size_t)n_sys * n_sys);
    int32_t* gt = (int32_t*)mxMalloc(sizeof(int32_t) * 3 * (size_t)n_sys);
    check(smg_classify(n_sys, Mx, My, Mzv, gt), NULL);
    mwSize dims[2] = {(mwSize)n_sys, 3};
    plhs[0] = mxCreateNumericArray(2, dims, mxDOUBLE_CLASS, mxREAL);
    double* out = mxGetPr(plhs[0]);
    for (int j = 0; j < n_sys; ++j)
        for (int k = 0; k < 3; ++k) out[j + (size_t)k * n_sys] = gt[3 * j + k];
    mxFree(gt);
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    if (nrhs >= 1 && mxIsChar(prhs[0])) {
        char mode[16];
        if (mxGetString(prhs[0], mode, sizeof mode) != 0 || strcmp(mode, "classify") != 0)
            mexErrMsgIdAndTxt("starmap:gpu:usage", "unknown mode (the only one is 'classify')");
        classify(nlhs, plhs, nrhs, prhs);
        return;
    }
    if (nrhs != 4 || nlhs > 2)
        mexErrMsgIdAndTxt("starmap:gpu:usage", "usage: [U, ms] = starmap_solver_mex(desc, U0, dt, nsteps)");
    const mxArray* d = prhs[0];
    if (!mxIsStruct(d) || mxGetNumberOfElements(d) != 1)
        mexErrMsgIdAndTxt("starmap:gpu:desc", "desc must be a 1x1 struct");

    smg_problem p;
    memset(&p, 0, sizeof p);
    const mxArray* Mz = desc_field(d, "Mz");
    const int n_sys = (int)mxGetM(Mz);
    if (n_sys < 1 || mxGetN(Mz) != (size_t)n_sys) mexErrMsgIdAndTxt("starmap:gpu:desc", "'Mz' must be square");
    p.n_sys = n_sys;
    const double* nv = dbl(desc_field(d, "n"), "n", 3);
    const double* bcv = dbl(desc_field(d, "bc"), "bc", 3);
    const double* hv = dbl(desc_field(d, "h"), "h", 3);
    for (int k = 0; k < 3; ++k) {
        p.n[k] = whole(nv[k], 1, 1 << 30, "n");
        p.bc[k] = whole(bcv[k], 0, 1, "bc");
        p.h[k] = hv[k];
    }
    p.Mx = dbl(desc_field(d, "Mx"), "Mx", (size_t)n_sys * n_sys);
    p.My = dbl(desc_field(d, "My"), "My", (size_t)n_sys * n_sys);
    p.Mz = dbl(Mz, "Mz", (size_t)n_sys * n_sys);

    /* grid types: MATLAB n_sys x 3 column-major -> gt[3*j + d] */
    const double* gtv = dbl(desc_field(d, "gt"), "gt", (size_t)n_sys * 3);
    int32_t* gt = (int32_t*)mxMalloc(sizeof(int32_t) * 3 * (size_t)n_sys);
    for (int j = 0; j < n_sys; ++j)
        for (int k = 0; k < 3; ++k) gt[3 * j + k] = whole(gtv[j + (size_t)k * n_sys], 1, 2, "gt");
    p.gt = gt;

    /* coefficient fields */
    const mxArray* fc = desc_field(d, "fields");
    if (!mxIsCell(fc)) mexErrMsgIdAndTxt("starmap:gpu:desc", "'fields' must be a cell array");
    const int nf = (int)mxGetNumberOfElements(fc);
    const double* fg = dbl(desc_field(d, "field_grid"), "field_grid", (size_t)nf * 3);
    smg_field* fields = (smg_field*)mxMalloc(sizeof(smg_field) * (size_t)(nf > 0 ? nf : 1));
    for (int f = 0; f < nf; ++f) {
        const mxArray* a = mxGetCell(fc, (size_t)f);
        if (!a) mexErrMsgIdAndTxt("starmap:gpu:desc", "field %d is empty", f + 1);
        const double* v = dbl(a, "fields{k}", 0);
        const size_t ne = mxGetNumberOfElements(a);
        if (ne == 0) mexErrMsgIdAndTxt("starmap:gpu:desc", "field %d is empty", f + 1);
        fields[f].data = ne == 1 ? NULL : v;
        fields[f].scalar = ne == 1 ? v[0] : 0.0;
        for (int k = 0; k < 3; ++k) fields[f].grid[k] = whole(fg[f + (size_t)k * nf], 1, 2, "field_grid");
    }
    p.n_fields = nf;
    p.fields = fields;
    p.sigma_t = index_table(d, "sigma_t", n_sys, nf);
    p.decay_t = index_table(d, "decay_t", n_sys, nf);
    p.source = index_table(d, "source", n_sys, nf);
    p.sigma_a = whole(mxGetScalar(desc_field(d, "sigma_a")), 1, nf, "sigma_a") - 1;
    p.decay_a = whole(mxGetScalar(desc_field(d, "decay_a")), 1, nf, "decay_a") - 1;
    p.filter_mode = whole(mxGetScalar(desc_field(d, "filter_mode")), 0, 2, "filter_mode");
    if (p.filter_mode != SMG_FILTER_NONE) p.filter1 = index_table(d, "filter1", n_sys, nf);
    if (p.filter_mode == SMG_FILTER_SUBSTEP) p.filter2 = index_table(d, "filter2", n_sys, nf);

    /* state: each component's element count against its staggered extents */
    const mxArray* U0 = prhs[1];
    if (!mxIsCell(U0) || mxGetNumberOfElements(U0) != (size_t)n_sys)
        mexErrMsgIdAndTxt("starmap:gpu:state", "U0 must be a cell array of %d components", n_sys);
    const double** Uin = (const double**)mxMalloc(sizeof(double*) * (size_t)n_sys);
    for (int j = 0; j < n_sys; ++j) {
        const mxArray* a = mxGetCell(U0, (size_t)j);
        size_t want = 1;
        for (int k = 0; k < 3; ++k) want *= (size_t)(p.n[k] + (gt[3 * j + k] == 2 && p.bc[k] == 1 ? 1 : 0));
        if (!a || !mxIsDouble(a) || mxIsComplex(a) || mxIsSparse(a) || mxGetNumberOfElements(a) != want)
            mexErrMsgIdAndTxt("starmap:gpu:state", "U0{%d} must be a real full double array of %d elements (U0{j})",
                              j + 1, (int)want);
        Uin[j] = mxGetPr(a);
    }
    const double dt = mxGetScalar(prhs[2]);
    const double nsd = mxGetScalar(prhs[3]);
    if (!(dt > 0)) mexErrMsgIdAndTxt("starmap:gpu:usage", "dt must be positive");
    if (!(nsd >= 0) || nsd != (double)(int64_t)nsd)
        mexErrMsgIdAndTxt("starmap:gpu:usage", "nsteps must be a whole number >= 0");

    smg_handle* h = NULL;
    check(smg_create(&p, &h), NULL);
    check(smg_set_state(h, Uin), h);
    check(smg_set_dt(h, dt), h);
    check(smg_run(h, (int64_t)nsd), h);

    /* outputs with the sizes of the inputs */
    plhs[0] = mxCreateCellMatrix(1, (size_t)n_sys);
    double** Uout = (double**)mxMalloc(sizeof(double*) * (size_t)n_sys);
    for (int j = 0; j < n_sys; ++j) {
        const mxArray* src = mxGetCell(U0, (size_t)j);
        mxArray* dst = mxCreateNumericArray(mxGetNumberOfDimensions(src), mxGetDimensions(src), mxDOUBLE_CLASS,
                                            mxREAL);
        Uout[j] = mxGetPr(dst);
        mxSetCell(plhs[0], (size_t)j, dst);
    }
    check(smg_get_state(h, Uout), h);
    double ms = 0.0;
    int64_t launches = 0;
    if (nsd > 0) check(smg_last_run_stats(h, &ms, &launches), h);
    smg_destroy(h);
    if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(ms);
    mxFree(Uout);
    mxFree(Uin);
    mxFree((void*)p.filter2);
    mxFree((void*)p.filter1);
    mxFree((void*)p.source);
    mxFree((void*)p.decay_t);
    mxFree((void*)p.sigma_t);
    mxFree(fields);
    mxFree(gt);
}
