function sys = fame_q_system(N,E,P,q)
%FAME_Q_SYSTEM Mass and null-space-free basis handles of the B200 library for one Bloch
% point: the device-side counterpart of exp1/build_experiment1_q_system.m.  E is the real
% permittivity gpuArray on the (2N)^6 grid (column-major, exp1/build_experiment1_common.m),
% P the 6x3 cut matrix and q the Bloch vector.  The reference's operator fields (W1, W2,
% invC, V blocks) stay on the device inside the handles.
    sys=struct('N',N,'NF',(2*N)^6);
    sys.fame.mass=fame_mex('mass_create',N,E);
    sys.fame.basis=fame_mex('basis_create',N,P,q(:));
end
