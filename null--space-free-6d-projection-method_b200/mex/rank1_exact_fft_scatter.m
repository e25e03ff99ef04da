function Xfft = rank1_exact_fft_scatter(x,plan)
%RANK1_EXACT_FFT_SCATTER Drop-in for exp1/rank1_exact_fft_scatter.m on libfame_b200:
% the length-plan.M DFT of x (NF x nrhs complex double gpuArray) embedded at
% plan.inputIdx, computed by the library's mixed-radix kernels.

    if isvector(x), x=x(:); end
    if size(x,1)~=plan.NF
        error('rank1_exact_fft_scatter:BadSize','x must have plan.NF rows.');
    end
    Xfft=fame_mex('rank1_exact_fft_scatter',complex(gpuArray(x)),plan);
end
