function o = airt_solver_opts(o, lbound, ubound, stoprule, taudelta, res_dims, dk)
%AIRT_SOLVER_OPTS  Fields shared by the sirt/art/cart option structs of
%   airt_mex: bounds, stopping rule code (0 NONE, 1 DP, 2 ME, 3 NCP, as
%   check_stoprules.m names them), taudelta and the NCP shape.  The inputs
%   are check_inputs.m's outputs.
o.lbound = lbound;
o.ubound = ubound;
switch upper(stoprule)
    case 'NONE', o.stoprule = 0;
    case 'DP',   o.stoprule = 1;
    case 'ME',   o.stoprule = 2;
    case 'NCP',  o.stoprule = 3;
    otherwise,   error('The chosen stopping rule is not valid.');
end
if ~isnan(taudelta)
    o.taudelta = taudelta;
end
if o.stoprule == 3
    o.res_dims = res_dims;
    o.ncp_smooth = numel(dk);   % check_inputs keeps dk = inf(ncp_smooth,1)
end
end
