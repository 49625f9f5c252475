// dq_fft.cu — spectrum of the ensemble-averaged dipole correlation.
//
// Replaces spectraClass::singleSpectraCalc's cuFFT Z2Z INVERSE
// (spectraClass.cu:621-626; plan at initLibs.cu:60-70): an in-place radix-2
// decimation-in-time inverse DFT, X_k = sum_j x_j exp(+2 pi i jk/n),
// unnormalised (the reference applies its mu_tot^2 / totalSteps scaling on
// the host, spectraClass.cu:641-690).  The correlation is zero-padded to the
// requested power-of-two length first.  Spectra are computed once per run,
// so log2(n) small launches are ample.
#include "dq_internal.h"

namespace dq {

__global__ void k_fft_load(int n_in, int len, double inv_traj, const cd* __restrict__ corr, cd* __restrict__ x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) {
        // bit-reversed placement
        int lg = 31 - __clz(len);
        int r = __brev(i) >> (32 - lg);
        x[r] = (i < n_in) ? cscale(corr[i], inv_traj) : cmk(0.0, 0.0);
    }
}

__global__ void k_fft_pass(int len, int half, cd* __restrict__ x) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < len / 2; t += gridDim.x * blockDim.x) {
        int g = t / half, k = t - g * half;
        int i = g * 2 * half + k, j = i + half;
        double s, c;
        sincospi((double)k / (double)half, &s, &c);   // exp(+i pi k / half)
        cd w = cmk(c, s);
        cd u = x[i], v = cmul(x[j], w);
        x[i] = cadd(u, v);
        x[j] = csub(u, v);
    }
}

// out = IDFT_len(scale * in[0..n_in), zero-padded); len a power of two.
dq_status fft_inverse(dq_ctx* c, int len, const cd* in, int n_in, double scale, cd* out) {
    int blocks = std::max(1, std::min(148 * 4, (len + 255) / 256));
    k_fft_load<<<blocks, 256, 0, c->stream>>>(std::min(n_in, len), len, scale, in, out);
    for (int half = 1; half < len; half <<= 1) k_fft_pass<<<blocks, 256, 0, c->stream>>>(len, half, out);
    return check_cuda(c, cudaGetLastError(), "inverse DFT");
}

dq_status spectrum(dq_ctx* c, int len, cd* d_out) {
    return fft_inverse(c, len, c->d_corr, c->steps_done + 1, 1.0 / c->cfg.n_traj, d_out);
}

}  // namespace dq

extern "C" dq_status dq_get_spectrum(dq_ctx* c, int len, dq_cdouble* out) {
    using namespace dq;
    if (!c || !out) return DQ_ERR_ARG;
    if (len < 2 || (len & (len - 1)) != 0) {
        c->err = "spectrum: length must be a power of two >= 2";
        return DQ_ERR_ARG;
    }
    if (c->last_path == 1 && c->bat) {
        dq_status st = batched_collect_corr(c);
        if (st) return st;
    }
    cd* d = nullptr;
    dq_status st = check_cuda(c, cudaMalloc(&d, sizeof(cd) * (size_t)len), "spectrum alloc");
    if (st) return st;
    st = spectrum(c, len, d);
    if (!st) st = check_cuda(c, cudaMemcpyAsync(out, d, sizeof(cd) * (size_t)len, cudaMemcpyDeviceToHost, c->stream),
                             "spectrum copy");
    if (!st) st = check_cuda(c, cudaStreamSynchronize(c->stream), "spectrum sync");
    cudaFree(d);
    return st;
}
