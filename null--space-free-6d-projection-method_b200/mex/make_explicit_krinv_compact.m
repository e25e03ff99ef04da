function [KrInvOp,getStats] = make_explicit_krinv_compact(sys,tolCG,maxitCG,budget) %#ok<INUSD>
%MAKE_EXPLICIT_KRINV_COMPACT K_r^{-1} on the B200 library (same signature as the reference's
% exp1/make_explicit_krinv_compact.m).  sys.fame holds the handles made by fame_q_system:
% sys.fame.basis (fame_mex 'basis_create') and sys.fame.mass (fame_mex 'mass_create').
% sys.fame.opts may set prec_mode (1 = mixed) and mhatPreconditioner (0 = the reference's
% plain pcg, whose iteration counts getStats then reproduces).
    if nargin<2 || isempty(tolCG), tolCG=1e-10; end
    if nargin<3 || isempty(maxitCG), maxitCG=1200; end
    opts=struct('tolCG',tolCG,'maxitCG',maxitCG);
    if isfield(sys.fame,'opts')
        f=fieldnames(sys.fame.opts);
        for j=1:numel(f), opts.(f{j})=sys.fame.opts.(f{j}); end
    end
    h=fame_mex('krinv_create',sys.fame.basis,sys.fame.mass,0,opts);
    KrInvOp=@(q) fame_mex('krinv_apply',h,q);
    getStats=@() fame_mex('krinv_stats',h);
end
