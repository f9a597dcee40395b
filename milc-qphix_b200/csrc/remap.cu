// Layout remap between MILC's raw arrays and the device field layouts (K6),
// and precision conversion of link sets.
//
// Reference: QPHIX_F3_create_V_from_raw / extract_V_to_raw
// (qphix_f3.cpp:63-159, 474-543) and asqtad_create_L_from_raw /
// extract_L_to_raw (qphix_f3.cpp:954-1070, 1086-1192).  The raw order inside
// a parity block is the device block order, so the remap is a pure
// transpose (AoS reals -> component-major complex) plus the split of the
// 4 link families into the 16-matrix block of each output parity.
#include <cstring>

#include "device_common.cuh"

namespace qb {

template <typename S, typename RAW>
__global__ void k_vec_from_raw(VecView<S> d, const RAW *raw)
{
    using A = typename Acc<S>::type;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.vh) return;
    A v[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) v[i] = (A)raw[6 * (size_t)j + i];
    d.store(j, v);
}

template <typename S, typename RAW>
__global__ void k_vec_to_raw(RAW *raw, VecView<S> s)
{
    using A = typename Acc<S>::type;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= s.vh) return;
    A v[6];
    s.load(j, v);
#pragma unroll
    for (int i = 0; i < 6; ++i) raw[6 * (size_t)j + i] = (RAW)v[i];
}

template <typename S, typename RAW>
static void vfr(const Launch &L, VecBlock d, const void *raw)
{
    k_vec_from_raw<S, RAW><<<grid_for(L.g->vh), kBlock, 0, L.stream>>>(view<S>(d, L.g->vh),
                                                                        static_cast<const RAW *>(raw));
}

template <typename S, typename RAW>
static void vtr(const Launch &L, void *raw, VecBlock s)
{
    k_vec_to_raw<S, RAW><<<grid_for(L.g->vh), kBlock, 0, L.stream>>>(static_cast<RAW *>(raw),
                                                                      view<S>(s, L.g->vh));
}

void vec_from_raw(Prec p, VecBlock dst, const void *raw_dev, bool raw_double, const Launch &L)
{
    if (raw_double) {
        switch (p) {
        case Prec::Double: vfr<double, double>(L, dst, raw_dev); break;
        case Prec::Single: vfr<float, double>(L, dst, raw_dev); break;
        case Prec::Half: vfr<__half, double>(L, dst, raw_dev); break;
        }
    } else {
        switch (p) {
        case Prec::Double: vfr<double, float>(L, dst, raw_dev); break;
        case Prec::Single: vfr<float, float>(L, dst, raw_dev); break;
        case Prec::Half: vfr<__half, float>(L, dst, raw_dev); break;
        }
    }
}

void vec_to_raw(Prec p, void *raw_dev, bool raw_double, VecBlock src, const Launch &L)
{
    if (raw_double) {
        switch (p) {
        case Prec::Double: vtr<double, double>(L, raw_dev, src); break;
        case Prec::Single: vtr<float, double>(L, raw_dev, src); break;
        case Prec::Half: vtr<__half, double>(L, raw_dev, src); break;
        }
    } else {
        switch (p) {
        case Prec::Double: vtr<double, float>(L, raw_dev, src); break;
        case Prec::Single: vtr<float, float>(L, raw_dev, src); break;
        case Prec::Half: vtr<__half, float>(L, raw_dev, src); break;
        }
    }
}

// ------------------------------------------------------------------ links --
// complex numbers per 16-byte chunk of each precision's link block
inline int link_k(Prec p) { return p == Prec::Double ? 1 : (p == Prec::Single ? 2 : 4); }

// one thread per (raw site, dir, complex element) of one raw link family
// (slot s); raw reads are coalesced
template <typename D, typename RAW>
__global__ void k_links_from_raw(D *blk0, D *blk1, const RAW *raw, int slot, int vh, int k)
{
    const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t total = (size_t)2 * vh * 36;
    if (idx >= total) return;
    const int e = idx % 9;
    const int d = (idx / 9) % 4;
    const size_t s = idx / 36;
    const int cb = s >= (size_t)vh;
    const int j = (int)(s - (size_t)cb * vh);
    D *blk = cb ? blk1 : blk0;
    D z;
    z.x = raw[2 * idx];
    z.y = raw[2 * idx + 1];
    blk[link_cx_index(k, d, 9 * slot + e, j, vh)] = z;
}

template <typename S, typename RAW>
__global__ void k_links_to_raw(RAW *raw, const S *blk0, const S *blk1, int slot, int vh, int k)
{
    const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t total = (size_t)2 * vh * 36;
    if (idx >= total) return;
    const int e = idx % 9;
    const int d = (idx / 9) % 4;
    const size_t s = idx / 36;
    const int cb = s >= (size_t)vh;
    const int j = (int)(s - (size_t)cb * vh);
    const S *blk = cb ? blk1 : blk0;
    const S z = blk[link_cx_index(k, d, 9 * slot + e, j, vh)];
    raw[2 * idx] = (RAW)z.x;
    raw[2 * idx + 1] = (RAW)z.y;
}

static int grid_links(int vh) { return (int)(((size_t)2 * vh * 36 + kBlock - 1) / kBlock); }

void links_from_raw(Prec p, LinkSet &ls, const void *raw_dev, bool raw_double, int slot, const Launch &L)
{
    const int vh = L.g->vh;
    const int grid = grid_links(vh);
    const int k = link_k(p);
    if (p == Prec::Double) {
        if (raw_double)
            k_links_from_raw<double2, double><<<grid, kBlock, 0, L.stream>>>(
                (double2 *)ls.blk[0], (double2 *)ls.blk[1], (const double *)raw_dev, slot, vh, k);
        else
            k_links_from_raw<double2, float><<<grid, kBlock, 0, L.stream>>>(
                (double2 *)ls.blk[0], (double2 *)ls.blk[1], (const float *)raw_dev, slot, vh, k);
    } else if (p == Prec::Single) {
        if (raw_double)
            k_links_from_raw<float2, double><<<grid, kBlock, 0, L.stream>>>(
                (float2 *)ls.blk[0], (float2 *)ls.blk[1], (const double *)raw_dev, slot, vh, k);
        else
            k_links_from_raw<float2, float><<<grid, kBlock, 0, L.stream>>>(
                (float2 *)ls.blk[0], (float2 *)ls.blk[1], (const float *)raw_dev, slot, vh, k);
    }
}

void links_to_raw(Prec p, void *raw_dev, bool raw_double, const LinkSet &ls, int slot, const Launch &L)
{
    const int vh = L.g->vh;
    const int grid = grid_links(vh);
    const int k = link_k(p);
    if (p == Prec::Double) {
        if (raw_double)
            k_links_to_raw<double2, double><<<grid, kBlock, 0, L.stream>>>(
                (double *)raw_dev, (const double2 *)ls.blk[0], (const double2 *)ls.blk[1], slot, vh, k);
        else
            k_links_to_raw<double2, float><<<grid, kBlock, 0, L.stream>>>(
                (float *)raw_dev, (const double2 *)ls.blk[0], (const double2 *)ls.blk[1], slot, vh, k);
    } else if (p == Prec::Single) {
        if (raw_double)
            k_links_to_raw<float2, double><<<grid, kBlock, 0, L.stream>>>(
                (double *)raw_dev, (const float2 *)ls.blk[0], (const float2 *)ls.blk[1], slot, vh, k);
        else
            k_links_to_raw<float2, float><<<grid, kBlock, 0, L.stream>>>(
                (float *)raw_dev, (const float2 *)ls.blk[0], (const float2 *)ls.blk[1], slot, vh, k);
    }
}

// max |component| per family (fat: slots 0,1; Naik: slots 2,3) over both
// parity blocks, for the 16-bit fixed-point ranges
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_absmax(const S *b0, const S *b1, int vh, int k, unsigned int *out)
{
    float m[2] = {0.f, 0.f};
    const size_t n = (size_t)4 * 36 * vh;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int d = (int)(i / ((size_t)36 * vh));
        const size_t r = i % ((size_t)36 * vh);
        const int c = (int)(r / vh);
        const int j = (int)(r % vh);
        const size_t at = link_cx_index(k, d, c, j, vh);
        const S a = b0[at], e = b1[at];
        const int f = (c / 9) >= 2;
        m[f] = fmaxf(m[f], fmaxf(fmaxf(fabsf((float)a.x), fabsf((float)a.y)), fmaxf(fabsf((float)e.x), fabsf((float)e.y))));
    }
    for (int f = 0; f < 2; ++f) {
        float v = m[f];
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0) atomicMax(out + f, __float_as_uint(v));  // v >= 0: uint order = float order
    }
}

void links_absmax(Prec p, const LinkSet &src, LinkSet &dst, const Launch &L, double *scratch)
{
    unsigned int *d = reinterpret_cast<unsigned int *>(scratch);
    cudaMemsetAsync(d, 0, 2 * sizeof(unsigned int), L.stream);
    const int grid = 148 * 8;
    if (p == Prec::Double)
        k_absmax<double2><<<grid, kBlock, 0, L.stream>>>((const double2 *)src.blk[0], (const double2 *)src.blk[1], L.g->vh, 1, d);
    else
        k_absmax<float2><<<grid, kBlock, 0, L.stream>>>((const float2 *)src.blk[0], (const float2 *)src.blk[1], L.g->vh, 2, d);
    unsigned int h[2] = {0, 0};
    cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, L.stream);
    cudaStreamSynchronize(L.stream);
    for (int f = 0; f < 2; ++f) {
        float v;
        memcpy(&v, &h[f], sizeof(v));
        dst.link_max[f] = v;
    }
}

// precision conversion between link blocks (each in its own chunking)
template <typename D, typename S>
__global__ void k_links_convert(D *dst, int kd, const S *src, int ks, int vh, float inv_fat, float inv_long)
{
    const size_t n = (size_t)4 * 36 * vh;
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int d = (int)(i / ((size_t)36 * vh));
    const size_t r = i % ((size_t)36 * vh);
    const int c = (int)(r / vh);
    const int j = (int)(r % vh);
    const S z = src[link_cx_index(ks, d, c, j, vh)];
    D q;
    if constexpr (std::is_same<D, short2>::value) {
        // offset binary u = q + 32768 (see fx16x2 in device_common.cuh)
        const float inv = (c / 9) >= 2 ? inv_long : inv_fat;
        q.x = (short)(unsigned short)(__float2int_rn((float)z.x * inv) + 32768);
        q.y = (short)(unsigned short)(__float2int_rn((float)z.y * inv) + 32768);
    } else {
        q.x = z.x;
        q.y = z.y;
    }
    dst[link_cx_index(kd, d, c, j, vh)] = q;
}

void links_convert(Prec dst_p, LinkSet &dst, Prec src_p, const LinkSet &src, const Launch &L)
{
    const int vh = L.g->vh;
    const size_t n = (size_t)4 * 36 * vh;
    const int grid = (int)((n + kBlock - 1) / kBlock);
    const float inv_fat = dst.link_max[0] > 0 ? 32767.0f / dst.link_max[0] : 0.f;
    const float inv_long = dst.link_max[1] > 0 ? 32767.0f / dst.link_max[1] : 0.f;
    const int kd = link_k(dst_p), ks = link_k(src_p);
    for (int cb = 0; cb < 2; ++cb) {
        if (dst_p == Prec::Single && src_p == Prec::Double)
            k_links_convert<float2, double2><<<grid, kBlock, 0, L.stream>>>((float2 *)dst.blk[cb], kd, (const double2 *)src.blk[cb], ks, vh, 0.f, 0.f);
        else if (dst_p == Prec::Double && src_p == Prec::Single)
            k_links_convert<double2, float2><<<grid, kBlock, 0, L.stream>>>((double2 *)dst.blk[cb], kd, (const float2 *)src.blk[cb], ks, vh, 0.f, 0.f);
        else if (dst_p == Prec::Half && src_p == Prec::Double)
            k_links_convert<short2, double2><<<grid, kBlock, 0, L.stream>>>((short2 *)dst.blk[cb], kd, (const double2 *)src.blk[cb], ks, vh, inv_fat, inv_long);
        else if (dst_p == Prec::Half && src_p == Prec::Single)
            k_links_convert<short2, float2><<<grid, kBlock, 0, L.stream>>>((short2 *)dst.blk[cb], kd, (const float2 *)src.blk[cb], ks, vh, inv_fat, inv_long);
    }
}

}  // namespace qb
