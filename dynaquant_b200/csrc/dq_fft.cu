// dq_fft.cu — spectrum of the ensemble-averaged dipole correlation.
//
// Replaces spectraClass::singleSpectraCalc's cuFFT Z2Z INVERSE
// (spectraClass.cu:621-626; plan at initLibs.cu:60-70): an in-place radix-2
// decimation-in-time inverse DFT, X_k = sum_j x_j exp(+2 pi i jk/n),
// unnormalised (the reference applies its mu_tot^2 / totalSteps scaling on
// the host, spectraClass.cu:641-690).  The correlation is zero-padded to the
// requested power-of-two length first.  Spectra are computed once per run,
// so log2(n) small launches are ample.
#include <algorithm>
#include <cmath>

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

// gpuSpectraHelper.cu:16-42: the correlation point k is dressed with a
// Gaussian of time dt (k + 1) (the reference's offset by one) for k < n_dress
__global__ void k_dress(int n_dress, double sigma, double dt, cd* __restrict__ x) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_dress; k += gridDim.x * blockDim.x) {
        const double t = dt * (k + 1);
        const double g = exp(-0.5 * (t / sigma) * (t / sigma));
        x[k] = cscale(x[k], g);
    }
}

dq_status dress_correlation(dq_ctx* c, int n_dress, cd* x) {
    if (!(c->dress_sigma > 0.0) || n_dress <= 0) return DQ_OK;
    k_dress<<<std::max(1, std::min(148 * 4, (n_dress + 255) / 256)), 256, 0, c->stream>>>(n_dress, c->dress_sigma,
                                                                                       c->cfg.dt, x);
    return check_cuda(c, cudaGetLastError(), "line-shape dressing");
}

// the ensemble-mean correlation (dressed when set), zero-padded to len, inverse DFT
dq_status spectrum(dq_ctx* c, int len, cd* d_out, cd* d_tmp) {
    const int np = c->steps_done + 1;
    dq_status st = check_cuda(c, cudaMemcpyAsync(d_tmp, c->d_corr, sizeof(cd) * np, cudaMemcpyDeviceToDevice,
                                                 c->stream), "spectrum copy");
    if (!st) st = dress_correlation(c, c->steps_done, d_tmp);
    if (!st) st = fft_inverse(c, len, d_tmp, np, 1.0 / observed_trajectories(c), d_out);
    return st;
}

}  // namespace dq

extern "C" dq_status dq_get_spectrum(dq_ctx* c, int len, dq_cdouble* out) {
    dq::DeviceScope dev_scope(c);
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
    dq_status st = check_cuda(c, cudaMalloc(&d, sizeof(cd) * ((size_t)len + c->steps_done + 1)), "spectrum alloc");
    if (st) return st;
    st = spectrum(c, len, d, d + len);
    if (!st) st = check_cuda(c, cudaMemcpyAsync(out, d, sizeof(cd) * (size_t)len, cudaMemcpyDeviceToHost, c->stream),
                             "spectrum copy");
    if (!st) st = check_cuda(c, cudaStreamSynchronize(c->stream), "spectrum sync");
    cudaFree(d);
    return st;
}

extern "C" dq_status dq_set_line_dressing(dq_ctx* c, double sigma_fs) {
    dq::DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (!(sigma_fs >= 0.0) || !std::isfinite(sigma_fs)) {
        c->err = "line_dressing: sigma must be >= 0 (0 turns the dressing off)";
        return DQ_ERR_ARG;
    }
    c->dress_sigma = sigma_fs;
    return DQ_OK;
}
