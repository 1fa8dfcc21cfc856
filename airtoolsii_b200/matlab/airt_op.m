classdef airt_op < handle
%AIRT_OP  Owner of a libairt problem handle (a GPU system matrix or a
%   matrix-free projector).  The handle is freed when the last reference to
%   the object goes away, e.g. when an operator closure made by
%   paralleltomo/fanlineartomo in this directory is cleared.
    properties (SetAccess = private)
        h   % uint64 handle of airt_mex
    end
    methods
        function obj = airt_op(h)
            obj.h = h;
        end
        function delete(obj)
            if ~isempty(obj.h)
                airt_mex('destroy', obj.h);
                obj.h = [];
            end
        end
    end
end
