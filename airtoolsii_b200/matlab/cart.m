function [X,info] = cart(cart_method,varargin)
%CART  Column-action (CART) sweeps on the GPU (libairt, B200).
%
%   [X,info] = cart(cart_method,A,b,K)
%   [X,info] = cart(cart_method,A,b,K,x0)
%   [X,info] = cart(cart_method,A,b,K,x0,options)
%
%   Drop-in for AIR Tools II cart/cart.m with the same arguments, outputs
%   and messages.  check_inputs and calc_relaxpar are the toolbox's own; the
%   column norms, the sweeps with flagging/unflagging (THR, Kbegin,
%   Nunflag), the box projection and the stopping rule run in libairt.
%   The unflagging draws come from libairt's counter-based generator
%   (options.seed, default 0), not from MATLAB's randi stream.

t_total = tic;
if isempty(cart_method)
    cart_method = 'columnaction';
end
[~,b,~,n,K,kmax,x0,lbound,ubound,stoprule,taudelta,relaxparinput, ...
    ~,res_dims,~,dk,~,verbose,damp,THR,Kbegin,Nunflag] = check_inputs(varargin{:});
relaxpar = calc_relaxpar(relaxparinput);
[h, keep] = airt_handle(varargin{1}); %#ok<ASGLU>

o = struct('relaxpar', relaxpar, 'damp', damp, 'THR', THR, 'Kbegin', Kbegin, ...
    'Nunflag', Nunflag, 'seed', 0);
if nargin > 5 && isstruct(varargin{5}) && isfield(varargin{5}, 'seed')
    o.seed = varargin{5}.seed;
end
if ischar(cart_method)
    if ~strcmpi(cart_method, 'columnaction')
        error('Unknown CART method specified')
    end
    o.order_kind = 0;
else
    o.order_kind = 2;
    o.cols = cart_method(:);
end
o = airt_solver_opts(o, lbound, ubound, stoprule, taudelta, res_dims, dk);
[X, g] = airt_mex('cart', h, o, b, x0, K);

info.stoprule = g.stoprule;
info.finaliter = g.finaliter;
info.relaxpar = relaxpar;
K = K(:);
info.itersaved = [K(K<info.finaliter); info.finaliter];
info.timetaken = toc(t_total);
if verbose
    airt_verbose(verbose, kmax, g.resnorms, relaxpar, info.timetaken);
end
end
