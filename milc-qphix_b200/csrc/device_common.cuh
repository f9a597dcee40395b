// Device helpers shared by the kernels: field loads/stores for every
// storage precision, SU(3) arithmetic, and the deterministic grid reduction
// that finishes in the last block.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "internal.h"

namespace qb {

constexpr int kBlock = 256;        // threads per block of the site kernels
constexpr int kMaxPartials = 1 << 16;

// accumulation type of a storage type
template <typename S> struct Acc { using type = float; };
template <> struct Acc<double> { using type = double; };

// ---------------------------------------------------------------- vectors --
template <typename S> struct VecView;

template <> struct VecView<double> {
    double2 *p;
    int vh;
    __device__ __forceinline__ void load(int j, double v[6]) const {
        const double2 a = __ldg(p + j), b = __ldg(p + vh + j), c = __ldg(p + 2 * vh + j);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
    }
    __device__ __forceinline__ void load_cg(int j, double v[6]) const {
        const double2 a = __ldcg(p + j), b = __ldcg(p + vh + j), c = __ldcg(p + 2 * vh + j);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
    }
    __device__ __forceinline__ void store(int j, const double v[6]) const {
        p[j] = make_double2(v[0], v[1]);
        p[vh + j] = make_double2(v[2], v[3]);
        p[2 * vh + j] = make_double2(v[4], v[5]);
    }
};

template <> struct VecView<float> {
    float2 *p;
    int vh;
    __device__ __forceinline__ void load(int j, float v[6]) const {
        const float2 a = __ldg(p + j), b = __ldg(p + vh + j), c = __ldg(p + 2 * vh + j);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
    }
    __device__ __forceinline__ void load_cg(int j, float v[6]) const {
        const float2 a = __ldcg(p + j), b = __ldcg(p + vh + j), c = __ldcg(p + 2 * vh + j);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
    }
    __device__ __forceinline__ void store(int j, const float v[6]) const {
        p[j] = make_float2(v[0], v[1]);
        p[vh + j] = make_float2(v[2], v[3]);
        p[2 * vh + j] = make_float2(v[4], v[5]);
    }
};

// 16-bit fixed point is stored in offset binary, u = q + 32768 in [1, 65535].
// Two values of a 32-bit word become floats without the conversion pipe
// (I2F, an eighth of the FP32 rate, bounded the 16-bit Dslash): PRMT places
// u in the mantissa of 2^23 (0x4B000000 | u = 2^23 + u exactly) and one FADD
// removes 2^23 + 32768, leaving q exactly.
__device__ __forceinline__ float2 fx16x2(unsigned w)
{
    return make_float2(__int_as_float(__byte_perm(w, 0x4B000000u, 0x7610)) - 8421376.0f,
                       __int_as_float(__byte_perm(w, 0x4B000000u, 0x7632)) - 8421376.0f);
}

// 16-bit storage: per-site norm = max |component| of the site (float), each
// component stored as 16-bit fixed point q = round(32767 v / norm).  Inside a
// normalised site fixed point keeps 15 bits where FP16 keeps 11.  A site is
// one 16-byte record {u0|u1, u2|u3, u4|u5, norm} with u = q + 32768.
template <> struct VecView<__half> {
    int4 *p;
    int vh;
    static __device__ __forceinline__ void unpack(const int4 w, float v[6]) {
        const float n = __int_as_float(w.w) * (1.0f / 32767.0f);
        const unsigned q[3] = {(unsigned)w.x, (unsigned)w.y, (unsigned)w.z};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float2 f = fx16x2(q[k]);
            v[2 * k] = f.x * n;
            v[2 * k + 1] = f.y * n;
        }
    }
    __device__ __forceinline__ void load(int j, float v[6]) const { unpack(__ldg(p + j), v); }
    __device__ __forceinline__ void load_cg(int j, float v[6]) const { unpack(__ldcg(p + j), v); }
    // Stores v and replaces it by the value a later load returns, so callers
    // never read back what they just wrote (a read-only-path load of data
    // written by the same kernel is not coherent).
    __device__ __forceinline__ void store(int j, float v[6]) const {
        float m = 0.f;
#pragma unroll
        for (int k = 0; k < 6; ++k) m = fmaxf(m, fabsf(v[k]));
        const float inv = m > 0.f ? 32767.0f / m : 0.f;
        const float n = m * (1.0f / 32767.0f);
        int q[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            q[k] = __float2int_rn(v[k] * inv);
            v[k] = (float)q[k] * n;
        }
        p[j] = make_int4((int)((unsigned)(q[0] + 32768) | ((unsigned)(q[1] + 32768) << 16)),
                         (int)((unsigned)(q[2] + 32768) | ((unsigned)(q[3] + 32768) << 16)),
                         (int)((unsigned)(q[4] + 32768) | ((unsigned)(q[5] + 32768) << 16)), __float_as_int(m));
    }
};

template <typename S> __host__ __device__ inline VecView<S> view(VecBlock b, int vh);
template <> __host__ __device__ inline VecView<double> view<double>(VecBlock b, int vh) {
    return VecView<double>{static_cast<double2 *>(b.data), vh};
}
template <> __host__ __device__ inline VecView<float> view<float>(VecBlock b, int vh) {
    return VecView<float>{static_cast<float2 *>(b.data), vh};
}
template <> __host__ __device__ inline VecView<__half> view<__half>(VecBlock b, int vh) {
    return VecView<__half>{static_cast<int4 *>(b.data), vh};
}

// ------------------------------------------------------------------ links --
// Streaming loads (evict-first): every link is used once per Dslash, so
// links must not displace the gathered colour vectors from L1/L2.
// Layout: see link_cx_index (internal.h).  Each precision loads whole
// 16-byte chunks, as many per batch as the arithmetic that follows needs, so
// a thread keeps 150-300 bytes of loads in flight.

template <typename S> struct LinkView;

// FP64: one matrix (9 double2 chunks) at a time
template <> struct LinkView<double> {
    const double2 *p;
    int vh;
    __device__ __forceinline__ void load_mat(int d, int s, int j, double u[18]) const {
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const double2 z = __ldcs(p + link_cx_index(1, d, 9 * s + e, j, vh));
            u[2 * e] = z.x; u[2 * e + 1] = z.y;
        }
    }
};

// FP32: a forward/backward pair (slots 2h, 2h+1) is 18 complex = 9 float4
template <> struct LinkView<float> {
    const float4 *p;
    int vh;
    // the 9 chunks of pair h of direction d, left packed: the pipelined
    // Dslash issues them one stage ahead and unpacks them when it uses them
    __device__ __forceinline__ void fetch_pair(int d, int h, int j, float4 c[9]) const {
        const float4 *q = p + ((size_t)d * 18 + 9 * h) * vh + j;
#pragma unroll
        for (int k = 0; k < 9; ++k) c[k] = __ldcs(q + (size_t)k * vh);
    }
};

// 16-bit fixed point: value = q * link_max / 32767 with one range for the fat
// slots and one for the Naik slots; all four matrices of a direction are
// 36 complex = 9 chunks of 16 bytes
template <> struct LinkView<__half> {
    const int4 *p;
    int vh;
    float scale_fat, scale_long;
    __device__ __forceinline__ void load_quad(int d, int j, int4 raw[9]) const {
        const int4 *q = p + (size_t)d * 9 * vh + j;
#pragma unroll
        for (int c = 0; c < 9; ++c) raw[c] = __ldcs(q + (size_t)c * vh);
    }
    // the fixed-point integers q of slot s out of the raw chunks
    // (offset-binary 16-bit values, two per word: slot s is words 9s .. 9s+8);
    // the link is q * scale_fat (slots 0, 1) or q * scale_long (slots 2, 3)
    __device__ __forceinline__ static void unpack_q(const int4 raw[9], int s, float u[18]) {
        const unsigned *w = reinterpret_cast<const unsigned *>(raw);
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const float2 f = fx16x2(w[9 * s + k]);
            u[2 * k] = f.x;
            u[2 * k + 1] = f.y;
        }
    }
};

// FP32 fat links and Naik links without their third rows (layout: internal.h,
// LinkSet::recon): the loads shared by the 12-real and 13-real forms
struct ReconLinks {
    const float4 *p;
    int vh;
    // raw chunks of the fat forward/backward pair (9) and of rows 0-1 of the
    // Naik forward and backward links (6) of direction d, left packed so the
    // pipelined Dslash can issue them one stage ahead
    __device__ __forceinline__ void fetch_fat(int d, int j, float4 c[9]) const {
        const float4 *q = p + (size_t)d * kReconChunks * vh + j;
#pragma unroll
        for (int k = 0; k < 9; ++k) c[k] = __ldcs(q + (size_t)k * vh);
    }
    __device__ __forceinline__ void fetch_naik(int d, int j, float4 c[6]) const {
        const float4 *q = p + ((size_t)d * kReconChunks + 9) * vh + j;
#pragma unroll
        for (int k = 0; k < 6; ++k) c[k] = __ldcs(q + (size_t)k * vh);
    }
    // rows 0-1 of the forward (uf) and backward (ub) Naik links
    __device__ __forceinline__ static void unpack_naik(const float4 c[6], float uf[18], float ub[18]) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            uf[4 * k] = c[k].x; uf[4 * k + 1] = c[k].y; uf[4 * k + 2] = c[k].z; uf[4 * k + 3] = c[k].w;
            ub[4 * k] = c[3 + k].x; ub[4 * k + 1] = c[3 + k].y; ub[4 * k + 2] = c[3 + k].z; ub[4 * k + 3] = c[3 + k].w;
        }
    }
    // (cr, ci)_k = (row0 x row1)_k: (a x b)_k = a_{k+1} b_{k+2} - a_{k+2} b_{k+1}
    __device__ __forceinline__ static void cross01(const float u[18], int k, float &cr, float &ci) {
        const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        const float ar1 = u[2 * k1], ai1 = u[2 * k1 + 1], ar2 = u[2 * k2], ai2 = u[2 * k2 + 1];
        const float br1 = u[6 + 2 * k1], bi1 = u[6 + 2 * k1 + 1], br2 = u[6 + 2 * k2], bi2 = u[6 + 2 * k2 + 1];
        cr = (ar1 * br2 - ai1 * bi2) - (ar2 * br1 - ai2 * bi1);
        ci = (ar1 * bi2 + ai1 * br2) - (ar2 * bi1 + ai2 * br1);
    }
    // row 2 = f * conj(row0 x row1), f real
    __device__ __forceinline__ static void rebuild(float u[18], float f) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float cr, ci;
            cross01(u, k, cr, ci);
            u[12 + 2 * k] = f * cr;
            u[12 + 2 * k + 1] = -f * ci;  // conjugate
        }
    }
    // row 2 = (lr + i li) * conj(row0 x row1)
    __device__ __forceinline__ static void rebuild(float u[18], float lr, float li) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float cr, ci;
            cross01(u, k, cr, ci);
            u[12 + 2 * k] = lr * cr + li * ci;
            u[12 + 2 * k + 1] = li * cr - lr * ci;
        }
    }
};

// 12-real: lambda = sign * scale, one magnitude for the field
template <> struct LinkView<Recon12> : ReconLinks {
    const unsigned *sign;
    float scale;
    static constexpr bool has_lam = false;
    __device__ __forceinline__ unsigned fetch_aux(int j) const { return __ldg(sign + j); }
    __device__ __forceinline__ float4 fetch_lam(int, int) const { return make_float4(0.f, 0.f, 0.f, 0.f); }
    // the Naik forward (uf) and backward (ub) links of direction d from their
    // chunks, third rows rebuilt
    __device__ __forceinline__ void naik_from(const float4 c[6], int d, unsigned bits, float4, float uf[18],
                                              float ub[18]) const {
        unpack_naik(c, uf, ub);
        rebuild(uf, (bits >> (2 * d)) & 1u ? -scale : scale);
        rebuild(ub, (bits >> (2 * d + 1)) & 1u ? -scale : scale);
    }
};

// 13-real: a complex lambda per link, (forward, backward) of direction d in
// one float4
template <> struct LinkView<Recon13> : ReconLinks {
    const float4 *lam;
    static constexpr bool has_lam = true;
    __device__ __forceinline__ unsigned fetch_aux(int) const { return 0u; }
    __device__ __forceinline__ float4 fetch_lam(int d, int j) const { return __ldcs(lam + (size_t)d * vh + j); }
    __device__ __forceinline__ void naik_from(const float4 c[6], int, unsigned, float4 l, float uf[18],
                                              float ub[18]) const {
        unpack_naik(c, uf, ub);
        rebuild(uf, l.x, l.y);
        rebuild(ub, l.z, l.w);
    }
};

// ------------------------------------------------------------------ SU(3) --
// acc += U v
template <typename A>
__device__ __forceinline__ void mv_add(A acc[6], const A u[18], const A v[6])
{
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const A ur = u[6 * r + 2 * c], ui = u[6 * r + 2 * c + 1];
            acc[2 * r] += ur * v[2 * c] - ui * v[2 * c + 1];
            acc[2 * r + 1] += ur * v[2 * c + 1] + ui * v[2 * c];
        }
    }
}

// acc -= U^dag v
template <typename A>
__device__ __forceinline__ void mv_adj_sub(A acc[6], const A u[18], const A v[6])
{
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            // (U^dag)_{rc} = conj(U_{cr})
            const A ur = u[6 * c + 2 * r], ui = u[6 * c + 2 * r + 1];
            acc[2 * r] -= ur * v[2 * c] + ui * v[2 * c + 1];
            acc[2 * r + 1] -= ur * v[2 * c + 1] - ui * v[2 * c];
        }
    }
}

// ------------------------------------------------------------- reductions --
// A finishing functor with `static constexpr bool kWarp = true` is called as
// fin(totals, lane) by all 32 lanes of one warp (per-shift work in parallel,
// with __syncwarp between dependent steps); others as fin(totals) by one
// thread.
template <typename F, typename = void> struct IsWarpFin : std::false_type {};
template <typename F> struct IsWarpFin<F, std::void_t<decltype(F::kWarp)>> : std::bool_constant<F::kWarp> {};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Reduce NV doubles over the grid.  Every block writes its partial sums to
// partials[i*gridDim.x + blockIdx.x]; the last block to arrive sums them in
// block order (deterministic) and calls fin(totals) from thread 0 -- or,
// when `split` is given (a domain-decomposed solve), stores the totals of
// this GPU in split->dd_red[] for the sum over GPUs, after which a
// one-thread kernel calls fin (k_dd_fin).
// Must be called by every thread of every block (uniform control flow).
template <int NV, typename F>
__device__ __forceinline__ void grid_reduce(double (&v)[NV], double *partials,
                                            unsigned int *counter, F fin, SolverState *split = nullptr)
{
    __shared__ double sm[NV][32];  // one slot per warp, any block size up to 1024
    __shared__ bool am_last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        v[i] = warp_sum(v[i]);
        if (lane == 0) sm[i][w] = v[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double s = 0;
            for (int k = 0; k < nw; ++k) s += sm[i][k];
            partials[i * gridDim.x + blockIdx.x] = s;
        }
        __threadfence();
        const unsigned int prev = atomicAdd(counter, 1u);
        am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    double t[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double s = 0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
            s += __ldcg(partials + i * gridDim.x + b);
        s = warp_sum(s);
        if (lane == 0) sm[i][w] = s;
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double s = 0;
            for (int k = 0; k < nw; ++k) s += sm[i][k];
            t[i] = s;  // every lane of warp 0 sums the same slots in the same order
        }
        if (split) {
            if (lane == 0)
#pragma unroll
                for (int i = 0; i < NV; ++i) split->dd_red[i] = t[i];
        } else if constexpr (IsWarpFin<F>::value) {
            fin(t, lane);
        } else if (lane == 0) {
            fin(t);
        }
        __syncwarp();
        if (lane == 0) {
            *counter = 0;
            __threadfence();
        }
    }
}

__device__ __forceinline__ double round_to(double v, int single) { return single ? (double)(float)v : v; }

// true when the chunk-local iteration `gate` was cancelled by an earlier stop
__device__ __forceinline__ bool gated_off(const SolverState *st, int gate)
{
    return gate >= 0 && gate > *(volatile const int *)&st->stop_at;
}

inline int grid_for(int n) { return (n + kBlock - 1) / kBlock; }

// Second half of a split reduction: after the totals in st->dd_red have been
// summed over the GPUs, one thread applies the reduction's finishing step.
// Gated like the reducing kernel.
template <int NV, typename Fin>
__global__ void k_dd_fin(SolverState *st, int gate, Fin fin)
{
    // launched with one warp
    if (threadIdx.x >= 32 || (gate >= 0 && gate > *(volatile const int *)&st->stop_at)) return;
    double t[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) t[i] = st->dd_red[i];
    if constexpr (IsWarpFin<Fin>::value) fin(t, (int)threadIdx.x);
    else if (threadIdx.x == 0) fin(t);
}

// Ends the device run of a solver phase: records the stopping iteration for
// the chunked launcher and, inside a CUDA-graph while loop, clears the loop
// condition.  Called by one thread.
__device__ __forceinline__ void stop_run(SolverState *st, int gate)
{
    st->stop_at = gate;
    if (st->use_cond) cudaGraphSetConditional(st->cond, 0);
}

// hard limits of one device run: the iteration cap and a failed kernel wait
__device__ __forceinline__ bool run_guard(const SolverState *st)
{
    return st->iteration >= st->iter_cap || (st->err && *(volatile int *)st->err);
}

// ------------------------------------------------- TMA bulk copies (sm_100a) --
// 1-D bulk copy global -> shared completing on an mbarrier (no multicast).
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order this thread's earlier generic-proxy shared accesses before later
// async-proxy (bulk copy) writes to shared memory
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                         uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// L2 eviction policy for data read exactly once (links)
__device__ __forceinline__ uint64_t policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// L2 eviction policy for data read again soon (the neighbour planes of the
// tile variant: every input plane is staged for nine output planes)
__device__ __forceinline__ uint64_t policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each poll may suspend the
// thread for a short, hardware-defined time) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit = 1u << 22)
{
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace qb
