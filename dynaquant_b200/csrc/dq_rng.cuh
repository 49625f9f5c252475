// dq_rng.cuh — counter-based noise for the stochastic site energies.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11) keyed by the 64-bit seed, with counter
// {site, step, traj/2, purpose<<24 | substep}; the two normals of a block
// belong to the even and the odd trajectory of the pair.  Uniforms become normals by
// Box-Muller; log, sin and cos are this file's own series (binary range
// reduction + atanh series for log, octant reduction + Taylor polynomials for
// sin/cos) evaluated with explicit fma and intrinsics that are never
// contracted, so every draw equals the host restatement's bit for bit.
//
// Replaces the reference's shared cuRAND MRG32k3a states
// (gpuSysHelper.cu:10-26, 53-62, 97-123), which up to ceil(N/4096) threads
// read and wrote back without synchronisation.
#pragma once
#include <cstdint>

namespace dq {

enum : uint32_t { P_OU = 1, P_GAUSS = 2, P_OU_INIT = 3, P_STATIC = 4, P_ZZPHASE = 5 };

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint32_t hi0 = __umulhi(0xD2511F53u, c[0]);
        uint32_t lo0 = 0xD2511F53u * c[0];
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]);
        uint32_t lo1 = 0xCD9E8D57u * c[2];
        uint32_t n0 = hi1 ^ c[1] ^ k0;
        uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    }
}

// 1/(2k+1), k = 0..11
__device__ __constant__ static const double kLogC[12] = {
    0x1.0000000000000p+0, 0x1.5555555555555p-2, 0x1.999999999999ap-3, 0x1.2492492492492p-3,
    0x1.c71c71c71c71cp-4, 0x1.745d1745d1746p-4, 0x1.3b13b13b13b14p-4, 0x1.1111111111111p-4,
    0x1.e1e1e1e1e1e1ep-5, 0x1.af286bca1af28p-5, 0x1.8618618618618p-5, 0x1.642c8590b2164p-5};
// (-1)^k/(2k+1)! and (-1)^k/(2k)!, k = 0..9
__device__ __constant__ static const double kSinC[10] = {
    0x1.0000000000000p+0, -0x1.5555555555555p-3, 0x1.1111111111111p-7, -0x1.a01a01a01a01ap-13,
    0x1.71de3a556c734p-19, -0x1.ae64567f544e4p-26, 0x1.6124613a86d09p-33, -0x1.ae7f3e733b81fp-41,
    0x1.952c77030ad4ap-49, -0x1.2f49b46814157p-57};
__device__ __constant__ static const double kCosC[10] = {
    0x1.0000000000000p+0, -0x1.0000000000000p-1, 0x1.5555555555555p-5, -0x1.6c16c16c16c17p-10,
    0x1.a01a01a01a01ap-16, -0x1.27e4fb7789f5cp-22, 0x1.1eed8eff8d898p-29, -0x1.93974a8c07c9dp-37,
    0x1.ae7f3e733b81fp-45, -0x1.6827863b97d97p-53};

// log of a positive normal double.
__device__ __forceinline__ double own_log(double x) {
    const double LN2_HI = 0x1.62e42fee00000p-1, LN2_LO = 0x1.a39ef35793c76p-33;
    const double SQRT2 = 0x1.6a09e667f3bcdp+0;
    unsigned long long b = __double_as_longlong(x);
    int e = (int)((b >> 52) & 0x7ff) - 1023;
    double f = __longlong_as_double((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (f > SQRT2) { f = __dmul_rn(f, 0.5); e += 1; }
    double s = __ddiv_rn(__dsub_rn(f, 1.0), __dadd_rn(f, 1.0));
    double z = __dmul_rn(s, s);
    double p = kLogC[11];
#pragma unroll
    for (int k = 10; k >= 0; --k) p = __fma_rn(p, z, kLogC[k]);
    double ls = __dmul_rn(__dadd_rn(s, s), p);
    double de = (double)e;
    return __fma_rn(de, LN2_HI, __fma_rn(de, LN2_LO, ls));
}

__device__ __forceinline__ void sincos_pio4(double g, double& s, double& c) {
    const double PIO4_HI = 0x1.921fb54442d18p-1, PIO4_LO = 0x1.1a62633145c07p-55;
    double x = __fma_rn(g, PIO4_HI, __dmul_rn(g, PIO4_LO));
    double y = __dmul_rn(x, x);
    double ps = kSinC[9];
#pragma unroll
    for (int k = 8; k >= 0; --k) ps = __fma_rn(ps, y, kSinC[k]);
    double pc = kCosC[9];
#pragma unroll
    for (int k = 8; k >= 0; --k) pc = __fma_rn(pc, y, kCosC[k]);
    s = __dmul_rn(x, ps);
    c = pc;
}

// sin and cos of 2 pi u, u in [0,1)
__device__ __forceinline__ void own_sincos_2pi(double u, double& S, double& C) {
    double t = __dmul_rn(u, 8.0);
    int k = (int)t;
    double f = __dsub_rn(t, (double)k);
    double sa, ca;
    sincos_pio4((k & 1) ? __dsub_rn(1.0, f) : f, sa, ca);
    switch (k & 7) {
        case 0: S = sa;  C = ca;  break;
        case 1: S = ca;  C = sa;  break;
        case 2: S = ca;  C = -sa; break;
        case 3: S = sa;  C = -ca; break;
        case 4: S = -sa; C = -ca; break;
        case 5: S = -ca; C = -sa; break;
        case 6: S = -ca; C = sa;  break;
        default: S = -sa; C = ca; break;
    }
}

// Both normals of one Philox block, keyed by the trajectory pair: z0 (cosine
// branch) belongs to trajectory 2*tpair, z1 (sine branch) to 2*tpair + 1.
__device__ __forceinline__ void normal_pair(uint64_t seed, uint32_t purpose, uint32_t tpair,
                                            uint32_t step, uint32_t site, uint32_t sub,
                                            double& z0, double& z1) {
    uint32_t c[4] = {site, step, tpair, (purpose << 24) | sub};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    unsigned long long a = ((unsigned long long)c[1] << 32) | c[0];
    unsigned long long b = ((unsigned long long)c[3] << 32) | c[2];
    double u1 = __dmul_rn((double)((a >> 11) + 1), 0x1.0p-53);
    double u2 = __dmul_rn((double)(b >> 11), 0x1.0p-53);
    double r = __dsqrt_rn(__dmul_rn(-2.0, own_log(u1)));
    double sn, cs;
    own_sincos_2pi(u2, sn, cs);
    z0 = __dmul_rn(r, cs);
    z1 = __dmul_rn(r, sn);
}

__device__ __forceinline__ double normal(uint64_t seed, uint32_t purpose, uint32_t traj, uint32_t step,
                                         uint32_t site, uint32_t sub) {
    double z0, z1;
    normal_pair(seed, purpose, traj >> 1, step, site, sub, z0, z1);
    return (traj & 1) ? z1 : z0;
}

// One Euler-Maruyama substep of the OU (Kubo-Anderson) offset in the
// reference's operation order (gpuSysHelper.cu:112):
// cur = cur - cur*invTau*subdt + coeff*xi*sqrt_subdt.
__device__ __forceinline__ double ou_substep(double cur, double inv_tau, double coeff, double subdt,
                                             double sqrt_subdt, double xi) {
    return __dadd_rn(__dsub_rn(cur, __dmul_rn(__dmul_rn(cur, inv_tau), subdt)),
                     __dmul_rn(__dmul_rn(coeff, xi), sqrt_subdt));
}

// `ns` OU substeps of one trajectory's offset.
__device__ __forceinline__ double ou_update(double cur, double inv_tau, double coeff, double subdt,
                                            double sqrt_subdt, int ns, uint64_t seed, uint32_t traj,
                                            uint32_t step, uint32_t site) {
    for (int s = 0; s < ns; ++s) {
        double z0, z1;
        normal_pair(seed, P_OU, traj >> 1, step, site, (uint32_t)s, z0, z1);
        cur = ou_substep(cur, inv_tau, coeff, subdt, sqrt_subdt, (traj & 1) ? z1 : z0);
    }
    return cur;
}

// `ns` OU substeps of the offsets of trajectories 2*tpair and 2*tpair + 1,
// one Philox block and one Box-Muller transform per substep.
__device__ __forceinline__ void ou_update_pair(double& c0, double& c1, double inv_tau, double coeff, double subdt,
                                               double sqrt_subdt, int ns, uint64_t seed, uint32_t tpair,
                                               uint32_t step, uint32_t site) {
    for (int s = 0; s < ns; ++s) {
        double z0, z1;
        normal_pair(seed, P_OU, tpair, step, site, (uint32_t)s, z0, z1);
        c0 = ou_substep(c0, inv_tau, coeff, subdt, sqrt_subdt, z0);
        c1 = ou_substep(c1, inv_tau, coeff, subdt, sqrt_subdt, z1);
    }
}

// ---- ZZ real noise (gpuSysHelper.cu:134-177) ------------------------------
// Phase fraction phi / 2 pi of oscillator osc at site for a trajectory, as a
// float: one Philox block per trajectory pair (even: first 64 bits).
__device__ __forceinline__ float zz_phase(uint64_t seed, uint32_t traj, uint32_t site, uint32_t osc) {
    uint32_t c[4] = {site, osc, traj >> 1, P_ZZPHASE << 24};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t a = (traj & 1) ? (((uint64_t)c[3] << 32) | c[2]) : (((uint64_t)c[1] << 32) | c[0]);
    float u = __double2float_rn(__dmul_rn((double)(a >> 11), 0x1.0p-53));
    if (u >= 1.0f) u = 0.0f;
    return u;
}

constexpr double kZZInv2Pi = 0x1.45f306dc9c883p-3;   // 1 / (2 pi)

// frac(omega t / 2 pi) for one oscillator at t = step dt
__device__ __forceinline__ double zz_wfrac(double omega, int step, double dt) {
    const double t = __dmul_rn((double)step, dt);
    const double w = __dmul_rn(__dmul_rn(omega, t), kZZInv2Pi);
    return __dsub_rn(w, floor(w));
}

// (c cos(omega t), c sin(omega t)) of one oscillator at t = step dt
__device__ __forceinline__ void zz_factors(double omega, double coeff, int step, double dt, double& ccw,
                                           double& csw) {
    double sw, cw;
    own_sincos_2pi(zz_wfrac(omega, step, dt), sw, cw);
    ccw = __dmul_rn(coeff, cw);
    csw = __dmul_rn(coeff, sw);
}

// acc + c cos(omega t + 2 pi u) as two fused multiply-adds
__device__ __forceinline__ double zz_acc(double acc, double ccw, double csw, float u) {
    double su, cu;
    own_sincos_2pi((double)u, su, cu);
    acc = __fma_rn(ccw, cu, acc);
    return __fma_rn(-csw, su, acc);
}

// the phases of trajectories 2 tpair and 2 tpair + 1 from one Philox block
__device__ __forceinline__ void zz_phase_pair(uint64_t seed, uint32_t tpair, uint32_t site, uint32_t osc, float& u0,
                                              float& u1) {
    uint32_t c[4] = {site, osc, tpair, P_ZZPHASE << 24};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t a = ((uint64_t)c[1] << 32) | c[0];
    const uint64_t b = ((uint64_t)c[3] << 32) | c[2];
    u0 = __double2float_rn(__dmul_rn((double)(a >> 11), 0x1.0p-53));
    u1 = __double2float_rn(__dmul_rn((double)(b >> 11), 0x1.0p-53));
    if (u0 >= 1.0f) u0 = 0.0f;
    if (u1 >= 1.0f) u1 = 0.0f;
}

struct ZZParams {
    int n_osc = 0;
    const double* omega = nullptr;   // rad/fs
    const double* coeff = nullptr;   // cm^-1
    double dt = 0.0;
};

}  // namespace dq

