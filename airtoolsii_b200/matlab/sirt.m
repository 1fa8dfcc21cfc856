function [X,info,ext_info] = sirt(sirt_method,varargin)
%SIRT  Simultaneous iterative reconstruction on the GPU (libairt, B200).
%
%   [X,info,ext_info] = sirt(sirt_method,A,b,K)
%   [X,info,ext_info] = sirt(sirt_method,A,b,K,x0)
%   [X,info,ext_info] = sirt(sirt_method,A,b,K,x0,options)
%
%   Drop-in for AIR Tools II sirt/sirt.m with the same arguments, outputs and
%   messages.  The toolbox's own check_inputs (input contract) and
%   calc_relaxpar (relaxation rule) run here; the weights M and D
%   (get_mfun_dfun.m), rho (calc_relaxpar.m:91-103), the iteration loop
%   (sirt.m:198-261) with its box projection and stopping rule run in
%   libairt through airt_mex.  A is a matrix or an operator made by this
%   directory's paralleltomo/fanlineartomo.  sirt_method is a method name
%   or a struct with fields M and D (vectors, diagonal or full matrices).

t_total = tic;
if isempty(sirt_method)
    sirt_method = 'sart';
end
[~,b,m,n,K,kmax,x0,lbound,ubound,stoprule,taudelta,relaxparinput, ...
    rho,res_dims,~,dk,~,verbose] = check_inputs(varargin{:});
[h, keep] = airt_handle(varargin{1}); %#ok<ASGLU> keep frees an uploaded matrix

o = airt_method_opts(sirt_method, m, n);
if ischar(sirt_method) && strcmpi(sirt_method, 'sart')
    rho = 1;                                   % sirt.m:166-168
end
if isnan(rho)
    rho = airt_mex('rho', h, o);
end
[relaxpar,casel,rho] = calc_relaxpar(relaxparinput,rho,kmax,[],n);

o.relax_kind = casel;
if casel == 1
    o.relaxpar = relaxpar;
elseif casel == 3
    o.relax_table = relaxpar(:);
end
o = airt_solver_opts(o, lbound, ubound, stoprule, taudelta, res_dims, dk);
[X, g] = airt_mex('sirt', h, o, b, x0, K);

info.stoprule = g.stoprule;
info.finaliter = g.finaliter;
if g.finaliter > 0
    info.relaxpar = g.relaxpar;
else
    info.relaxpar = relaxparinput;             % check_stoprules at k = 0
end
info.rho = rho;
K = K(:);
info.itersaved = [K(K<info.finaliter); info.finaliter];
info.timetaken = toc(t_total);
if verbose
    if casel == 1, lams = relaxpar; elseif casel == 3, lams = relaxpar; else, lams = nan; end
    airt_verbose(verbose, kmax, g.resnorms, lams, info.timetaken);
end

if nargout > 2
    if o.method == 5
        ext_info.M = o.M;  if isempty(o.M), ext_info.M = ones(m,1); end
        ext_info.D = o.D;  if isempty(o.D), ext_info.D = ones(n,1); end
    else
        [ext_info.M, ext_info.D] = airt_mex('weights', h, o.method);
    end
end
end

function o = airt_method_opts(sirt_method, m, n)
% Method code of airt_mex (0 landweber, 1 cimmino, 2 cav, 3 drop, 4 sart,
% 5 custom) and, for a custom struct, M and D as get_mfun_dfun.m:252-307
% reads them: vectors and diagonal matrices become diagonals, other
% matrices stay full.
o = struct();
if ischar(sirt_method)
    names = {'landweber','cimmino','cav','drop','sart'};
    code = find(strcmpi(sirt_method, names), 1) - 1;
    if isempty(code)
        error('SIRT method not defined.')
    end
    o.method = code;
elseif isstruct(sirt_method)
    o.method = 5;
    o.M = custom_weight(sirt_method, 'M', m);
    o.D = custom_weight(sirt_method, 'D', n);
else
    error(['First input must be a string with the SIRT method name or ',...
        'a struct with fields M and D characterizing a custom method.']);
end
end

function W = custom_weight(s, name, len)
W = [];
if ~isfield(s, name) || isempty(s.(name))
    return
end
W = s.(name);
if ~isnumeric(W)
    error('%s must be given as an array, either of dimension 0, 1 or 2.', name)
end
if isvector(W)
    W = full(double(W(:)));
elseif isdiag(W)
    W = full(double(diag(W)));
else
    W = full(double(W));
end
if (isvector(W) && numel(W) ~= len) || (~isvector(W) && any(size(W) ~= [len len]))
    error('%s has the wrong size.', name)
end
end
