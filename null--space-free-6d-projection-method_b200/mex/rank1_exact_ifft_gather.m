function y = rank1_exact_ifft_gather(Yfft,plan)
%RANK1_EXACT_IFFT_GATHER Drop-in for exp1/rank1_exact_ifft_gather.m on libfame_b200:
% ifft of Yfft (plan.M x nrhs complex double gpuArray) read at plan.targetIdx.

    if isvector(Yfft), Yfft=Yfft(:); end
    if size(Yfft,1)~=plan.M
        error('rank1_exact_ifft_gather:BadSize','Yfft must have plan.M rows.');
    end
    y=fame_mex('rank1_exact_ifft_gather',complex(gpuArray(Yfft)),plan);
end
