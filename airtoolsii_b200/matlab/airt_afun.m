function y = airt_afun(op, v, transp_flag)
%AIRT_AFUN  The afun interface of a libairt operator (the flags of
%   auxil/afun_matrix.m:44-53): 'notransp' -> A*v, 'transp' -> A'*v,
%   'size' -> [m n].  op is an airt_op.
switch transp_flag
    case 'size'
        y = airt_mex('size', op.h);
    case 'notransp'
        y = airt_mex('apply', op.h, full(double(v(:))), 0);
    case 'transp'
        y = airt_mex('apply', op.h, full(double(v(:))), 1);
    otherwise
        error('transp_flag must be ''notransp'', ''transp'' or ''size''.')
end
end
