function [A,b,x,theta,p,R,dw,sd] = fanlineartomo(N,theta,p,R,dw,sd,isDisp,isMatrix)
%FANLINEARTOMO  2D fan-beam tomography test problem (linear detector), on the GPU.
%
%   [A,b,x,theta,p,R,dw,sd] = fanlineartomo(N)
%   [A,b,x,theta,p,R,dw,sd] = fanlineartomo(N,theta,p,R,dw,sd,isDisp,isMatrix)
%
%   Drop-in for AIR Tools II testprobs/fanlineartomo.m with the same
%   arguments, defaults (theta = 0:2:358, p = round(sqrt(2)*N), R = 2,
%   dw = 2.5, sd = 3, the last three in units of N) and outputs.  The
%   detector element angles omega are formed here from the detector
%   positions; libairt traces the rays in FP64 on the GPU.  isMatrix = 0
%   returns a matrix-free operator handle as paralleltomo does.  isDisp is
%   ignored.

if nargin < 2 || isempty(theta), theta = 0:2:358; end
if nargin < 3 || isempty(p),     p = round(sqrt(2)*N); end
if nargin < 4 || isempty(R),     R = 2; end
if nargin < 5 || isempty(dw),    dw = 2.5; end
if nargin < 6 || isempty(sd),    sd = 3; end
if nargin < 8 || isempty(isMatrix), isMatrix = 1; end
theta = theta(:)';
R = R*N;  dw = dw*N;  sd = sd*N;
if R < sqrt(2)/2*N
    error('R must be greater than half squareroot 2')
end

% angle of every detector element seen from the source: element centres
% at multiples of dw/p from the detector centre (an element on the centre
% for odd p, half an element off it for even p)
dew = dw/p;
if mod(p,2)
    depos = (1:(p-1)/2)*dew;
    om = 90 - atand(sd./depos);
    omega = [-fliplr(om), 0, om];
else
    depos = ((1:p/2) - 0.5)*dew;
    om = 90 - atand(sd./depos);
    omega = [-fliplr(om), om];
end

h = airt_mex('fan', N, cosd(theta), sind(theta), cosd(omega), sind(omega), R, double(~isMatrix));
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
R = R/N;
end
