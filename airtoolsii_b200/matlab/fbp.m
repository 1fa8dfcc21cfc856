function x = fbp(A,b,theta,filter)
%FBP  Filtered back projection on the GPU (libairt).
%
%   x = fbp(A,b,theta)
%   x = fbp(A,b,theta,filter)
%
%   Drop-in for AIR Tools II auxil/fbp.m: filter is 'ram-lak' (default),
%   'shepp-logan', 'cosine', 'hamming', 'hann' or 'none'.  The frequency
%   response (the ramp n/max(n) on order = max(64, 2^nextpow2(2*nr))
%   samples, its first entry 0.4/order and last 1 - that, times the named
%   window, extended evenly) is built here; libairt convolves every
%   projection with its impulse response real(ifft(f)) in FP64, scales by
%   pi/(2*na) and back-projects with A'.

if nargin < 3
    error('Input A, b, theta must me specified')
end
if nargin < 4 || isempty(filter)
    filter = 'ram-lak';
end
[h, keep] = airt_handle(A); %#ok<ASGLU>
mn = airt_mex('size', h);
if strcmpi(filter, 'none')
    x = airt_mex('apply', h, full(double(b(:))), 1);
    return
end
na = numel(theta);
nr = mn(1)/na;
order = max(64, 2^nextpow2(2*nr));
n = 0:order/2;
f = n/max(n);
f(1) = 0.4/order;
f(end) = 1 - f(1);
w = 2*pi*n/order;
k = 2:numel(f);
switch lower(filter)
    case 'ram-lak'
    case 'shepp-logan'
        f(k) = f(k).*(sin(w(k)/2)./(w(k)/2));
    case 'cosine'
        f(k) = f(k).*cos(w(k)/2);
    case 'hamming'
        f(k) = f(k).*(0.54 + 0.46*cos(w(k)));
    case 'hann'
        f(k) = f(k).*(1 + cos(w(k)))/2;
    otherwise
        error('Iinvalid filter')
end
f = [f, f(end-1:-1:2)];
kernel = real(ifft(f));
x = airt_mex('fbp', h, full(double(b(:))), na, kernel(:));
end
