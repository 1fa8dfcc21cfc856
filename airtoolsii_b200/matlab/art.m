function [X,info] = art(art_method,varargin)
%ART  Algebraic reconstruction (Kaczmarz row sweeps) on the GPU (libairt).
%
%   [X,info] = art(art_method,A,b,K)
%   [X,info] = art(art_method,A,b,K,x0)
%   [X,info] = art(art_method,A,b,K,x0,options)
%
%   Drop-in for AIR Tools II art/art.m with the same arguments, outputs and
%   messages.  check_inputs and calc_relaxpar are the toolbox's own; the
%   row norms, the sweeps in the reference's row order (art.m:183-203,
%   227-285: kaczmarz, symkaczmarz with its last row applied twice, a
%   custom row vector, or randkaczmarz) and the stopping rule run in
%   libairt.  randkaczmarz draws its permutations and weighted rows here,
%   with MATLAB's own randperm/rand in the order the reference loop draws
%   them, and passes the rows to the GPU.  A function-handle relaxpar is
%   evaluated here at (k-1)*m + i for every row step i of sweep k
%   (art.m:273-275).

t_total = tic;
if isempty(art_method)
    art_method = 'kaczmarz';
end
[~,b,m,n,K,kmax,x0,lbound,ubound,stoprule,taudelta,relaxparinput, ...
    ~,res_dims,~,dk,~,verbose,damp] = check_inputs(varargin{:});
is_sym = ischar(art_method) && strncmpi(art_method, 'sym', 3);
if is_sym
    if any(mod(K,2))
        error('For symkaczmarz only even iteration numbers can be requested.');
    end
    K = K/2;
    kmax = kmax/2;
end
relaxpar = calc_relaxpar(relaxparinput);
[h, keep] = airt_handle(varargin{1}); %#ok<ASGLU>

o = struct('relaxpar', 1, 'damp', damp);
if isnumeric(relaxpar)
    o.relaxpar = relaxpar;
end
if ischar(art_method)
    switch lower(art_method)
        case 'kaczmarz',     o.order_kind = 0;
        case 'symkaczmarz',  o.order_kind = 1;
        case 'randkaczmarz', o.order_kind = 2;
        otherwise,           error('Unknown ART method specified')
    end
else
    o.order_kind = 2;
end

needs_rows = o.order_kind == 2 || isa(relaxparinput, 'function_handle');
if needs_rows
    % row norms on the device (the transposed products of art.m:161-181)
    normAi = row_norms(h, m);
    I = find(normAi > 0);
    if ~ischar(art_method)
        I = art_method(:)';
        I = I(normAi(I) > 0);
    elseif o.order_kind == 1
        I = [I, I(end:-1:1)];
    end
end
if o.order_kind == 2 && ischar(art_method)              % randkaczmarz
    w = normAi + damp*max(normAi);
    cumul = cumsum(w/sum(w));
    fast = norm(cumul - (1:m)/m, inf) < 0.05;
    rows = zeros(numel(I), kmax);
    loop_i = zeros(numel(I), kmax);
    for k = 1:kmax
        It = I(randperm(numel(I)));
        loop_i(:,k) = It(:);
        if fast
            rows(:,k) = It(:);
        else
            for t = 1:numel(It)
                rows(t,k) = sum(cumul < rand) + 1;
            end
        end
    end
    o.rows = rows(:);
    o.rows_stride = numel(I);
elseif o.order_kind == 2
    o.rows = I(:);
    loop_i = repmat(I(:), 1, kmax);
elseif needs_rows
    loop_i = repmat(I(:), 1, kmax);
end
if isa(relaxparinput, 'function_handle')
    tab = zeros(size(loop_i));
    for k = 1:kmax
        tab(:,k) = arrayfun(@(i) relaxparinput((k-1)*m + i), loop_i(:,k));
    end
    o.relax_table = tab(:);
end
o = airt_solver_opts(o, lbound, ubound, stoprule, taudelta, res_dims, dk);
if ~isempty(ubound) && any(isnan(ubound))                 % art.m:282 tests ~isnan
    o.ubound = [];
end
[X, g] = airt_mex('art', h, o, b, x0, K);

info.stoprule = g.stoprule;
info.finaliter = g.finaliter;
info.relaxpar = relaxpar;
if isnumeric(relaxpar) && g.finaliter > 0
    info.relaxpar = g.relaxpar;
end
if is_sym
    info.finaliter = 2*info.finaliter;
    K = 2*K;
end
K = K(:);
info.itersaved = [K(K<info.finaliter); info.finaliter];
info.timetaken = toc(t_total);
if verbose
    airt_verbose(verbose, kmax, g.resnorms, o.relaxpar, info.timetaken);
end
end

function normAi = row_norms(h, m)
% Squared row norms ||a_i||^2 of the stored matrix, as a 1 x m row.
A = airt_mex('export', h);
normAi = full(sum(A.^2, 2))';
if numel(normAi) ~= m
    error('AIRT:internal', 'row norm count mismatch')
end
end
