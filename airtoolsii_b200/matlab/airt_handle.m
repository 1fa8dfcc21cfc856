function [h, keep] = airt_handle(A)
%AIRT_HANDLE  libairt handle of the A argument of sirt/art/cart.
%   [h, keep] = airt_handle(A).  A is a matrix (uploaded for this call and
%   freed when KEEP, an airt_op, goes out of scope) or an operator closure
%   made by this directory's paralleltomo / fanlineartomo (whose handle is
%   reused).  libairt cannot call back into a general MATLAB function
%   handle, so any other function handle is an error.
if isa(A, 'function_handle')
    f = functions(A);
    if isfield(f, 'workspace') && ~isempty(f.workspace) && ...
            isfield(f.workspace{1}, 'op') && isa(f.workspace{1}.op, 'airt_op')
        keep = f.workspace{1}.op;
        h = keep.h;
        return
    end
    error('AIRT:operator', ['A must be a matrix or an operator made by ', ...
        'paralleltomo/fanlineartomo of the libairt toolbox directory.']);
end
if ~issparse(A)
    A = sparse(A);
end
h = airt_mex('matrix', double(A));
keep = airt_op(h);
end
