function output = starmap_solver(par)
%STARMAP_SOLVER  Drop-in for StaRMAP's starmap_solver (same call, same
%   output struct): the host setup runs here in MATLAB / GNU Octave, the
%   staggered-grid time loop runs on a B200 GPU through the MEX gateway
%   starmap_solver_mex (matlab/starmap_solver_mex.c, C ABI starmap_gpu.h).
%
%   output = starmap_solver(par)    with par = starmap_init(prob), as for the
%   reference (starmap_solver.m:1; starmap_init.m, the prob/par fields and
%   the closure matrices are used unchanged).
%
%   Steps, each restating the reference's semantics in this file's own code:
%     flags and moment orders ......................... starmap_solver.m:58-71
%     grid types (by the library's smg_classify) ...... starmap_solver.m:76-98
%     h, dt_hyp ....................................... starmap_solver.m:100-107
%     staggered coordinates and grids ................. starmap_solver.m:112-123
%     initial condition ............................... starmap_solver.m:140-146
%     first-step materials, dt, decay factors ......... starmap_solver.m:165-274
%     sources at t - dt/2, filters at the first step .. starmap_solver.m:276-305
%     the update loop (one MEX call per stretch
%     between output times) ........................... starmap_solver.m:307-421
%     output times by linear interpolation ............ starmap_solver.m:423-473
%     summary print and output struct ................. starmap_solver.m:476-500
%
%   Covered: autonomous problems (sigma_a, sigma_s0, sigma_sm, source and
%   filter hooks that do not take the time t) with the hyperbolic time step
%   (par.timestep = 0), any closure, 1D/2D/3D, both boundary conditions,
%   filters '', 'substep' and 'full'.  Other problems raise the error
%   starmap:gpu:unsupported; there is no CPU fallback.
%
%   This file and the gateway were written where neither MATLAB nor GNU
%   Octave is installed: the gateway is compiled and run against a test-only
%   stand-in of the MATLAB C API, fed with the descriptor this file builds,
%   and compared with the Python host's results; this file itself has not
%   been run.

t_start = tic;
n_sys = length(par.Mz);
% ---- flags (starmap_solver.m:58-71)
flag_filter = isfield(par,'filterfunction') && isfield(par,'f_position') && isfield(par,'mom_order');
if flag_filter
    f_mom_order = par.mom_order;
    f_position = par.f_position;
else
    f_position = '';
end
flag_ani = isfield(par,'sigma_sm') && isfield(par,'mom_order');
if flag_ani
    mom_order = par.mom_order;
else
    mom_order = [0 ones(1,n_sys-1)];
end
if ischar(par.mom_output) && strcmp(par.mom_output,'all'), par.mom_output = 1:n_sys; end
if isfield(par,'timestep') && par.timestep ~= 0
    error('starmap:gpu:unsupported', 'the GPU drop-in uses the hyperbolic time step (par.timestep = 0)');
end
if nargin(par.sigma_a) > 3 || nargin(par.sigma_s0) > 3 || (flag_ani && nargin(par.sigma_sm) > 4)
    error('starmap:gpu:unsupported', 'time-dependent materials are not supported by the GPU drop-in');
end
if ~isempty(par.source_ind) && nargin(par.source) >= 4
    error('starmap:gpu:unsupported', 'time-dependent sources are not supported by the GPU drop-in');
end
if flag_filter && nargin(par.filterfunction) > 6
    error('starmap:gpu:unsupported', 'time-dependent filters are not supported by the GPU drop-in');
end

% ---- grid types, spacing, time step (starmap_solver.m:76-107)
Mx = full(par.Mx); My = full(par.My); Mz = full(par.Mz);
gt = starmap_solver_mex('classify', Mx, My, Mz);        % n_sys x 3, entries 1 or 2
h = (par.ax([2 4 6]) - par.ax([1 3 5])) ./ par.n;
dt_hyp = min(h) / max(abs(eig(Mz)));
if par.n(1) ~= 1
    dt_hyp = dt_hyp/3;
elseif par.n(2) ~= 1
    dt_hyp = dt_hyp/2;
end

% ---- staggered coordinates (starmap_solver.m:112-118): the same colon
% ranges, so that hooks are sampled at identical points
crd = cell(3,2);
for d = 1:3
    a = par.ax(2*d-1); b = par.ax(2*d);
    crd{d,1} = a+h(d)/2:h(d):b-h(d)/2;
    crd{d,2} = a+h(d)*(1-par.bc(d)):h(d):b;
end
grids = containers.Map('KeyType','double','ValueType','any');
    function G = grid_of(g)                   % {X,Y,Z} of grid type g = [gx gy gz]
        key = g(1)*100 + g(2)*10 + g(3);
        if ~isKey(grids, key)
            [Xg,Yg,Zg] = ndgrid(crd{1,g(1)}, crd{2,g(2)}, crd{3,g(3)});
            grids(key) = {Xg,Yg,Zg};
        end
        G = grids(key);
    end
    function v = hook(fct, varargin)          % call with as many arguments as it takes
        v = fct(varargin{1:max(nargin(fct),1)});
    end
    function v = on_grid(val, G)              % scalar hook results stay scalars
        if isscalar(val), v = val; else, v = G{1}*0 + val; end
    end

% ---- initial condition (starmap_solver.m:140-146)
U = cell(1,n_sys);
for j = 1:n_sys
    G = grid_of(gt(j,:));
    U{j} = G{1}*0 + hook(par.ic, G{1}, G{2}, G{3}, j) * (nargin(par.ic) > 3 || j == 1);
end

% ---- first-step materials (starmap_solver.m:214-243), dt, decay factors
rows = unique([gt(2:end,:) mom_order(2:end)'], 'rows');     % (grid type, order) rows
G1 = grid_of([1 1 1]);
sA1 = on_grid(hook(par.sigma_a, G1{1}, G1{2}, G1{3}, 0), G1);
sT1 = cell(1, size(rows,1));
for r = 1:size(rows,1)
    G = grid_of(rows(r,1:3));
    sS = hook(par.sigma_s0, G{1}, G{2}, G{3}, 0);
    if flag_ani, sS = sS - hook(par.sigma_sm, G{1}, G{2}, G{3}, rows(r,4), 0); end
    sT1{r} = on_grid(hook(par.sigma_a, G{1}, G{2}, G{3}, 0) + sS, G);
end
dt = min(dt_hyp, par.tfinal/par.cn) * par.cn;              % starmap_solver.m:208
EA = expm1div(-sA1*dt/2);
ET = cellfun(@(s) expm1div(-s*dt/2), sT1, 'UniformOutput', false);

% ---- coefficient fields and the descriptor of starmap_solver_mex
fields = {}; field_grid = zeros(0,3);
    function k = add_field(v, g)
        fields{end+1} = v; field_grid(end+1,:) = g; k = numel(fields);
    end
sigma_t = zeros(1,n_sys); decay_t = zeros(1,n_sys);
row_of = @(j) find(ismember(rows, [gt(j,:) mom_order(j)], 'rows'), 1);
rt = zeros(1, size(rows,1)); re = rt;
for r = 1:size(rows,1)
    rt(r) = add_field(sT1{r}, rows(r,1:3));
    re(r) = add_field(ET{r}, rows(r,1:3));
end
ka = add_field(sA1, [1 1 1]);
ke = add_field(EA, [1 1 1]);
for j = 2:n_sys
    sigma_t(j) = rt(row_of(j)); decay_t(j) = re(row_of(j));
end
sigma_t(1) = ka; decay_t(1) = ke;                        % component 1 decays by sigma_a only
source = zeros(1,n_sys);
for j = par.source_ind                                    % sources at t - dt/2 (starmap_solver.m:276-282)
    G = grid_of(gt(j,:));
    source(j) = add_field(on_grid(hook(par.source, G{1}, G{2}, G{3}, dt-dt/2, j), G), gt(j,:));
end
filter_mode = 0; filter1 = zeros(1,n_sys); filter2 = zeros(1,n_sys);
if flag_filter && any(strcmp(f_position, {'substep','full'}))  % at the first step (starmap_solver.m:283-305)
    frows = unique([gt(2:end,:) f_mom_order(2:end)'], 'rows');
    filter_mode = 1 + strcmp(f_position, 'full');
    for r = 1:size(frows,1)
        G = grid_of(frows(r,1:3)); m = frows(r,4);
        members = find(ismember([gt f_mom_order(:)], frows(r,:), 'rows'))';
        members = members(members > 1);
        if filter_mode == 2
            k1 = add_field(on_grid(hook(par.filterfunction, par, dt, m, G{1}, G{2}, G{3}, dt), G), frows(r,1:3));
            filter1(members) = k1;
        else
            k1 = add_field(on_grid(hook(par.filterfunction, par, dt, m, G{1}, G{2}, G{3}, dt-dt/2), G), frows(r,1:3));
            k2 = add_field(on_grid(hook(par.filterfunction, par, dt, m, G{1}, G{2}, G{3}, dt), G), frows(r,1:3));
            filter1(members) = k1; filter2(members) = k2;
        end
    end
end
desc = struct('n', double(par.n), 'bc', double(par.bc), 'h', h, 'gt', gt, 'Mx', Mx, 'My', My, 'Mz', Mz, ...
              'fields', {fields}, 'field_grid', field_grid, 'sigma_t', sigma_t, 'decay_t', decay_t, ...
              'source', source, 'sigma_a', ka, 'decay_a', ke, 'filter_mode', filter_mode, ...
              'filter1', filter1, 'filter2', filter2);
t_setup = toc(t_start);

% ---- the loop (starmap_solver.m:162-421) with its output times (:423-473)
t_plot = [par.t_plot inf]; plot_count = 1;
t = 0; step_count = 0; t_gpu = 0; t_out = 0;
times = [];                                               % t after each step, overshoot included
while t < par.tfinal, t = t + dt; times(end+1) = t; end %#ok<AGROW>
done = 0;
while done < numel(times)
    % the next step whose end reaches an output time
    k = find(times(done+1:end) >= t_plot(plot_count) - 1e-14, 1);
    if isempty(k), k = numel(times) - done; end
    tic
    if k > 1, U = starmap_solver_mex(desc, U, dt, k-1); end
    Uprev = U(par.mom_output);
    U = starmap_solver_mex(desc, U, dt, 1);
    t_gpu = t_gpu + toc;
    done = done + k; t = times(done); step_count = done;
    tic
    while t >= t_plot(plot_count) - 1e-14
        lambda = (t_plot(plot_count) - t + dt)/dt;
        Uplot = cell(1, numel(par.mom_output));
        for q = 1:numel(par.mom_output)
            Uplot{q} = (1-lambda)*Uprev{q} + lambda*U{par.mom_output(q)};
        end
        par = call_output(par, Uplot, gt, crd, plot_count);
        plot_count = plot_count + 1;
    end
    t_out = t_out + toc;
end

% ---- summary and output struct (starmap_solver.m:476-500)
fprintf('%s with %s%s%d\n %d moments, %dx%dx%d grid, %0.0f time steps\n', par.name, par.closure_mod, ...
        par.closure, par.n_mom, n_sys, par.n, step_count)
ct = [t_gpu t_setup t_out];
ct = reshape([ct; ct/sum(ct)*1e2], 1, []);
fprintf(['CPU-times\n advection:%12.2fs%5.0f%%\n absorb/scatter:%7.2fs%5.0f%%\n ', ...
         'plotting:%13.2fs%5.0f%%\n'], ct)
if nargout
    xs = crd(1, gt(:,1)'); ys = crd(2, gt(:,2)'); zs = crd(3, gt(:,3)');
    switch par.dim
        case 1
            for j = 1:n_sys, U{j} = reshape(U{j}, length(zs{j}), []); end
            output = struct('x', zs, 'U', U);
        case 2
            for j = 1:n_sys, U{j} = reshape(U{j}, length(ys{j}), []); end
            output = struct('x', ys, 'y', zs, 'U', U);
        otherwise
            output = struct('x', xs, 'y', ys, 'z', zs, 'U', U);
    end
end
end

function par = call_output(par, Uplot, gt, crd, step)
% The output hook with the reference's arguments per dimension.
mo = par.mom_output;
xp = crd(1, gt(mo,1)'); yp = crd(2, gt(mo,2)'); zp = crd(3, gt(mo,3)');
switch par.dim
    case 1
        for q = 1:numel(Uplot), Uplot{q} = reshape(Uplot{q}, length(zp{q}), []); end
        if numel(mo) == 1, zp = zp{1}; Uplot = Uplot{1}; end
        args = {zp, Uplot};
    case 2
        for q = 1:numel(Uplot), Uplot{q} = reshape(Uplot{q}, length(yp{q}), []); end
        if numel(mo) == 1, yp = yp{1}; zp = zp{1}; Uplot = Uplot{1}; end
        args = {yp, zp, Uplot};
    otherwise
        if numel(mo) == 1, xp = xp{1}; yp = yp{1}; zp = zp{1}; Uplot = Uplot{1}; end
        args = {xp, yp, zp, Uplot};
end
if nargout(par.output)
    par = par.output(par, args{:}, step);
else
    par.output(par, args{:}, step);
end
end

function y = expm1div(x)
% (exp(x)-1)/x with the reference's branch: 1 + x/2 + x^2/6 for |x| <= 2e-4
% (starmap_solver.m:531-535).
y = 1 + x*.5 + x.^2/6;
big = abs(x) > 2e-4;
y(big) = (exp(x(big)) - 1)./x(big);
end
