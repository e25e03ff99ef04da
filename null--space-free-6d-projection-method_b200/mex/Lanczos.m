function [ev,ew,iter,info] = Lanczos(fncA,fncB,fncBinv,n,k,tol,maxiter,p,v0,flag_gpu,verbose) %#ok<INUSD>
%LANCZOS Restarted Lanczos of exp2/Lanczos.m on the B200 library: fncA must be a KrInvOp made
% by make_explicit_krinv_compact in this folder, and fncB = fncBinv = @(x) x (as in every call
% of the reference's hot path).  Returns the k largest theta of K_r^{-1} with their vectors.
    w=functions(fncA);
    if ~isfield(w,'workspace') || ~isfield(w.workspace{1},'h')
        error('Lanczos:BadInput','fncA must be a KrInvOp of make_explicit_krinv_compact (B200 library)');
    end
    x=gpuArray(complex(ones(4,1)));
    if ~isequal(fncB(x),x) || ~isequal(fncBinv(x),x)
        error('Lanczos:BadInput','only fncB = fncBinv = identity is supported');
    end
    if ~isa(v0,'gpuArray'), v0=gpuArray(v0); end
    [ev,ew,iter,info]=fame_mex('lanczos',w.workspace{1}.h,k,tol,maxiter,p,complex(v0));
end
