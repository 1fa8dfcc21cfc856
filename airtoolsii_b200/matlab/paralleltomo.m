function [A,b,x,theta,p,d] = paralleltomo(N,theta,p,d,isDisp,isMatrix)
%PARALLELTOMO  2D parallel-beam tomography test problem, built on the GPU.
%
%   [A,b,x,theta,p,d] = paralleltomo(N)
%   [A,b,x,theta,p,d] = paralleltomo(N,theta,p,d,isDisp,isMatrix)
%
%   Drop-in for AIR Tools II testprobs/paralleltomo.m with the same
%   arguments, defaults (theta = 0:179, p = round(sqrt(2)*N), d = p-1) and
%   outputs.  libairt traces the rays in FP64 on the GPU and returns the
%   same sparsity pattern as the reference's trace.  isMatrix = 1 gives the
%   sparse matrix A; isMatrix = 0 a matrix-free operator handle
%   A(v,'notransp'|'transp'|'size') that recomputes the rays on every
%   product and can be passed to sirt/art/cart of this directory (they then
%   run on it without copying a matrix).  isDisp (ray animation) is ignored.

if nargin < 2 || isempty(theta), theta = 0:179; end
if nargin < 3 || isempty(p),     p = round(sqrt(2)*N); end
if nargin < 4 || isempty(d),     d = p-1; end
if nargin < 6 || isempty(isMatrix), isMatrix = 1; end
theta = theta(:)';

offsets = linspace(-d/2, d/2, p);
h = airt_mex('parallel', N, cosd(theta), sind(theta), offsets, double(~isMatrix));
op = airt_op(h);
x = phantomgallery('shepplogan', N);
x = x(:);
if isMatrix
    A = airt_mex('export', h);
    b = A*x;
else
    A = @(v, transp_flag) airt_afun(op, v, transp_flag);
    b = A(x, 'notransp');
end
end
