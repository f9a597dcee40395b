// FP32 link sets with 12-real and 13-real Naik links.
//
// The reference can store the long (Naik) links without their third row
// (COMPRESSED_12 in asqtad_create_L_from_raw, qphix_f3.cpp:1008-1016) and
// rebuild it as conj(row0 x row1) with the staggered-phase sign
// (reconstruct_gauge_third_row, qphix_f3.cpp:1072-1084).  MILC's Naik links
// carry the Naik coefficient and the phases: a link c * U with U in U(3) and
// c real satisfies row2 = lambda * conj(row0 x row1) with lambda = det(U)/c.
// Two forms are kept here, both measured from the FP64 links:
//   12-real: U in SU(3) up to a sign (asqtad Naik links): lambda = sign * s
//            with one magnitude s for the field and a sign bit per link;
//   13-real: any U in U(3) (HISQ Naik links built from unitarised links):
//            lambda complex per link, stored as FP32.
// A field of neither form (a varying real factor, non-unitary links) is
// detected and keeps its 18-real links.  Only the FP32 copy used by the
// mixed-precision inner solve is compressed; FP64 links stay complete.
//
// Bytes per output site of the FP32 Dslash: 8 fat x 72 + 8 Naik x 48 + 48
// (vectors) + 4 (12-real sign word) = 1012 or + 64 (13-real ratios) = 1072,
// instead of 1200.
#include <algorithm>
#include <cmath>

#include "context.h"
#include "device_common.cuh"

namespace qb {

namespace {

constexpr int kProbeNV = 5;  // sums of the probe
constexpr int kProbeNM = 2;  // maxima of the probe

__device__ __forceinline__ void load_link64(const double2 *blk, int d, int slot, int j, int vh, double2 u[9])
{
#pragma unroll
    for (int e = 0; e < 9; ++e) u[e] = blk[link_cx_index(1, d, 9 * slot + e, j, vh)];
}

// c = conj(row0 x row1) of u
__device__ __forceinline__ void conj_cross(const double2 u[9], double2 c[3])
{
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        const double2 a1 = u[k1], a2 = u[k2], b1 = u[3 + k1], b2 = u[3 + k2];
        const double re = (a1.x * b2.x - a1.y * b2.y) - (a2.x * b1.x - a2.y * b1.y);
        const double im = (a1.x * b2.y + a1.y * b2.x) - (a2.x * b1.y + a2.y * b1.x);
        c[k] = make_double2(re, -im);
    }
}

// ratio rho = <c, row2> / |c|^2 of one Naik link (complex)
__device__ __forceinline__ double2 ratio(const double2 u[9], const double2 c[3], double *c2)
{
    double nr = 0, ni = 0, n2 = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double2 r = u[6 + k];
        nr += c[k].x * r.x + c[k].y * r.y;
        ni += c[k].x * r.y - c[k].y * r.x;
        n2 += c[k].x * c[k].x + c[k].y * c[k].y;
    }
    *c2 = n2;
    return n2 > 0 ? make_double2(nr / n2, ni / n2) : make_double2(0.0, 0.0);
}

// pass 0: sums of |rho|, (Im rho)^2, |row2 - Re(rho) c|^2, |row2|^2,
//         |row2 - rho c|^2, and the largest per-link relative residuals
//         |row2 - Re(rho) c| / |row2| and |row2 - rho c| / |row2|
// pass 1: sum of (|rho| - mean)^2 and the largest ||rho| - mean| / mean
// A field-wide RMS alone would let a few links whose rows rebuild to only
// ~1e-6 through; the maxima hold every link to the same bound.
__global__ void __launch_bounds__(kBlock) k_recon_probe(const double2 *blk, int vh, int pass, double mean,
                                                        double *partials)
{
    double s[kProbeNV] = {0, 0, 0, 0, 0};
    double mx[kProbeNM] = {0, 0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < vh * 8; t += gridDim.x * blockDim.x) {
        const int j = t >> 3, d = (t >> 1) & 3, slot = 2 + (t & 1);
        double2 u[9], c[3];
        load_link64(blk, d, slot, j, vh, u);
        conj_cross(u, c);
        double c2;
        const double2 rho = ratio(u, c, &c2);
        const double mag = fabs(rho.x);
        if (pass == 0) {
            double e_re = 0, e_cx = 0, n2 = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double dr = u[6 + k].x - rho.x * c[k].x, di = u[6 + k].y - rho.x * c[k].y;
                e_re += dr * dr + di * di;
                n2 += u[6 + k].x * u[6 + k].x + u[6 + k].y * u[6 + k].y;
                const double er = u[6 + k].x - (rho.x * c[k].x - rho.y * c[k].y);
                const double ei = u[6 + k].y - (rho.x * c[k].y + rho.y * c[k].x);
                e_cx += er * er + ei * ei;
            }
            s[0] += mag;
            s[1] += rho.y * rho.y;
            s[2] += e_re;
            s[3] += n2;
            s[4] += e_cx;
            // a link with a zero third row rebuilds only if row0 x row1 is zero too
            mx[0] = fmax(mx[0], n2 > 0 ? sqrt(e_re / n2) : (e_re > 0 ? 1.0 : 0.0));
            mx[1] = fmax(mx[1], n2 > 0 ? sqrt(e_cx / n2) : (e_cx > 0 ? 1.0 : 0.0));
        } else {
            s[0] += (mag - mean) * (mag - mean);
            mx[0] = fmax(mx[0], mean > 0 ? fabs(mag - mean) / mean : 1.0);
        }
    }
    __shared__ double sm[kProbeNV + kProbeNM][kBlock / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < kProbeNV; ++i) {
        const double v = warp_sum(s[i]);
        if (lane == 0) sm[i][w] = v;
    }
#pragma unroll
    for (int i = 0; i < kProbeNM; ++i) {
        double v = mx[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
        if (lane == 0) sm[kProbeNV + i][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < kProbeNV + kProbeNM) {
        const bool is_max = threadIdx.x >= kProbeNV;
        double v = 0;
        for (int k = 0; k < kBlock / 32; ++k) v = is_max ? fmax(v, sm[threadIdx.x][k]) : v + sm[threadIdx.x][k];
        partials[threadIdx.x * gridDim.x + blockIdx.x] = v;
    }
}

__global__ void k_sum_partials(const double *partials, int nb, double *out)
{
    const int i = threadIdx.x;
    if (i >= kProbeNV + kProbeNM) return;
    double v = 0;
    for (int b = 0; b < nb; ++b) v = i >= kProbeNV ? fmax(v, partials[i * nb + b]) : v + partials[i * nb + b];
    out[i] = v;
}

// FP32 blocks: per direction the fat pair (complex 0..17 -> 9 float4) and
// rows 0-1 of the Naik forward and backward links (12 complex -> 6 float4).
// MODE 1: sign bit 2d (forward) / 2d+1 (backward) when Re(rho) < 0;
// MODE 2: rho of the forward and backward Naik links of direction d as one
// float4 in lam[d*vh + j]
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_recon_pack(float4 *dst, unsigned *sign, float4 *lam, const double2 *blk,
                                                       int vh)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= vh) return;
    unsigned bits = 0;
#pragma unroll 1
    for (int d = 0; d < 4; ++d) {
        float4 *q = dst + (size_t)d * kReconChunks * vh + j;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            const double2 a = blk[link_cx_index(1, d, 2 * c, j, vh)];
            const double2 b = blk[link_cx_index(1, d, 2 * c + 1, j, vh)];
            q[(size_t)c * vh] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
        }
        double2 rh[2];
#pragma unroll
        for (int slot = 2; slot < 4; ++slot) {
            double2 u[9], c3[3];
            load_link64(blk, d, slot, j, vh, u);
            conj_cross(u, c3);
            double c2;
            rh[slot - 2] = ratio(u, c3, &c2);
            if (MODE == 1 && rh[slot - 2].x < 0) bits |= 1u << (2 * d + (slot - 2));
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                // rows 0-1 (6 complex) of this link: chunks 9 + 3*(slot-2) + c
                q[(size_t)(9 + 3 * (slot - 2) + c) * vh] =
                    make_float4((float)u[2 * c].x, (float)u[2 * c].y, (float)u[2 * c + 1].x, (float)u[2 * c + 1].y);
            }
        }
        if (MODE == 2)
            lam[(size_t)d * vh + j] = make_float4((float)rh[0].x, (float)rh[0].y, (float)rh[1].x, (float)rh[1].y);
    }
    if (MODE == 1) sign[j] = bits;
}

}  // namespace

int links_compress(LinkSet &dst, const LinkSet &src64, const Launch &L, double dev[5], int want)
{
    const int vh = L.g->vh;
    if (src64.prec != Prec::Double || !src64.valid) throw Error("links_compress: needs FP64 links");
    constexpr int NT = kProbeNV + kProbeNM;
    const int nb = 296;
    double *part = static_cast<double *>(dev_alloc(sizeof(double) * (NT * nb + NT)));
    double *sums = part + NT * nb;
    double h[NT], tot[NT] = {0, 0, 0, 0, 0, 0, 0};
    double mean = 0, spread = 0, spread_max = 0;
    for (int pass = 0; pass < 2; ++pass) {
        double acc[NT] = {0, 0, 0, 0, 0, 0, 0};
        for (int cb = 0; cb < 2; ++cb) {
            k_recon_probe<<<nb, kBlock, 0, L.stream>>>(static_cast<const double2 *>(src64.blk[cb]), vh, pass, mean,
                                                      part);
            k_sum_partials<<<1, 32, 0, L.stream>>>(part, nb, sums);
            QB_CUDA(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, L.stream));
            sync_check();
            for (int i = 0; i < kProbeNV; ++i) acc[i] += h[i];
            for (int i = kProbeNV; i < NT; ++i) acc[i] = std::max(acc[i], h[i]);
        }
        const double n = 2.0 * vh * 8;
        if (pass == 0) {
            for (int i = 0; i < NT; ++i) tot[i] = acc[i];
            mean = tot[0] / n;
        } else {
            spread = std::sqrt(acc[0] / n) / (mean > 0 ? mean : 1.0);
            spread_max = acc[kProbeNV];
        }
    }
    dev_free(part);
    const double n = 2.0 * vh * 8;
    dev[0] = mean;
    dev[1] = spread;
    dev[2] = mean > 0 ? std::sqrt(tot[1] / n) / mean : 1.0;
    dev[3] = tot[3] > 0 ? std::sqrt(tot[2] / tot[3]) : 1.0;
    dev[4] = tot[3] > 0 ? std::sqrt(tot[4] / tot[3]) : 1.0;
    // The rebuilt rows must be exact far below FP32 rounding, field-wide and
    // link by link: 12-real needs one magnitude for every link and a real
    // ratio rebuilding every third row; 13-real a complex ratio per link.
    const double max_re = tot[kProbeNV], max_cx = tot[kProbeNV + 1];
    const bool ok12 = mean > 0 && spread < 1e-9 && spread_max < 1e-9 && dev[2] < 1e-9 && dev[3] < 1e-9 &&
                      max_re < 1e-9;
    const bool ok13 = mean > 0 && dev[4] < 1e-9 && max_cx < 1e-9;
    int mode = 0;
    if (want == 1) mode = ok12 ? 1 : 0;
    else if (want == 2) mode = ok13 ? 2 : 0;
    else mode = ok12 ? 1 : (ok13 ? 2 : 0);
    if (!mode) return 0;
    dst = LinkSet{};
    for (int cb = 0; cb < 2; ++cb) {
        dst.blk[cb] = dev_alloc(sizeof(float4) * kReconChunks * 4 * (size_t)vh);
        const double2 *src = static_cast<const double2 *>(src64.blk[cb]);
        if (mode == 1) {
            dst.sign[cb] = dev_alloc(sizeof(unsigned) * (size_t)vh);
            k_recon_pack<1><<<grid_for(vh), kBlock, 0, L.stream>>>(
                static_cast<float4 *>(dst.blk[cb]), static_cast<unsigned *>(dst.sign[cb]), nullptr, src, vh);
        } else {
            dst.lam[cb] = dev_alloc(sizeof(float4) * 4 * (size_t)vh);
            k_recon_pack<2><<<grid_for(vh), kBlock, 0, L.stream>>>(static_cast<float4 *>(dst.blk[cb]), nullptr,
                                                                   static_cast<float4 *>(dst.lam[cb]), src, vh);
        }
    }
    QB_CUDA(cudaGetLastError());
    sync_check();
    dst.prec = Prec::Single;
    dst.recon = mode;
    dst.recon_scale = (float)mean;
    dst.valid = true;
    return mode;
}

}  // namespace qb
