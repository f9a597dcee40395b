// Device helpers shared by the kernels: field loads/stores for every
// storage precision, SU(3) arithmetic, and the deterministic grid reduction
// that finishes in the last block.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

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

// 16-bit storage: per-site norm = max |component| of the site (float), each
// component stored as 16-bit fixed point q = round(32767 v / norm).  Inside a
// normalised site fixed point keeps 15 bits where FP16 keeps 11.
template <> struct VecView<__half> {
    short2 *p;
    float *norm;
    int vh;
    __device__ __forceinline__ void load(int j, float v[6]) const {
        const float n = __ldg(norm + j) * (1.0f / 32767.0f);
        const short2 a = __ldg(p + j), b = __ldg(p + vh + j), c = __ldg(p + 2 * vh + j);
        v[0] = a.x * n; v[1] = a.y * n; v[2] = b.x * n; v[3] = b.y * n; v[4] = c.x * n; v[5] = c.y * n;
    }
    __device__ __forceinline__ void load_cg(int j, float v[6]) const {
        const float n = __ldcg(norm + j) * (1.0f / 32767.0f);
        const short2 a = __ldcg(p + j), b = __ldcg(p + vh + j), c = __ldcg(p + 2 * vh + j);
        v[0] = a.x * n; v[1] = a.y * n; v[2] = b.x * n; v[3] = b.y * n; v[4] = c.x * n; v[5] = c.y * n;
    }
    // Stores v and replaces it by the value a later load returns, so callers
    // never read back what they just wrote (a read-only-path load of data
    // written by the same kernel is not coherent).
    __device__ __forceinline__ void store(int j, float v[6]) const {
        float m = 0.f;
#pragma unroll
        for (int k = 0; k < 6; ++k) m = fmaxf(m, fabsf(v[k]));
        const float inv = m > 0.f ? 32767.0f / m : 0.f;
        const float n = m * (1.0f / 32767.0f);
        short q[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            q[k] = (short)__float2int_rn(v[k] * inv);
            v[k] = q[k] * n;
        }
        norm[j] = m;
        p[j] = make_short2(q[0], q[1]);
        p[vh + j] = make_short2(q[2], q[3]);
        p[2 * vh + j] = make_short2(q[4], q[5]);
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
    return VecView<__half>{static_cast<short2 *>(b.data), b.norm, vh};
}

// ------------------------------------------------------------------ links --
// Streaming loads (evict-first): every link is used once per Dslash, so
// links must not displace the gathered colour vectors from L1/L2.
template <typename S> struct LinkView;

template <> struct LinkView<double> {
    const double2 *p;
    int vh;
    __device__ __forceinline__ void load(int mat, int j, double u[18]) const {
        const double2 *q = p + (size_t)mat * 9 * vh + j;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const double2 z = __ldcs(q + (size_t)e * vh);
            u[2 * e] = z.x; u[2 * e + 1] = z.y;
        }
    }
};

template <> struct LinkView<float> {
    const float2 *p;
    int vh;
    __device__ __forceinline__ void load(int mat, int j, float u[18]) const {
        const float2 *q = p + (size_t)mat * 9 * vh + j;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const float2 z = __ldcs(q + (size_t)e * vh);
            u[2 * e] = z.x; u[2 * e + 1] = z.y;
        }
    }
};

// 16-bit fixed point links: value = q * link_max / 32767, one range for the
// fat slots (mat < 8) and one for the Naik slots
template <> struct LinkView<__half> {
    const short2 *p;
    int vh;
    float scale_fat, scale_long;
    __device__ __forceinline__ void load(int mat, int j, float u[18]) const {
        const short2 *q = p + (size_t)mat * 9 * vh + j;
        const float scale = mat < 8 ? scale_fat : scale_long;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const short2 z = __ldcs(q + (size_t)e * vh);
            u[2 * e] = z.x * scale; u[2 * e + 1] = z.y * scale;
        }
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
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Reduce NV doubles over the grid.  Every block writes its partial sums to
// partials[i*gridDim.x + blockIdx.x]; the last block to arrive sums them in
// block order (deterministic) and calls fin(totals) from thread 0.
// Must be called by every thread of every block (uniform control flow).
template <int NV, typename F>
__device__ __forceinline__ void grid_reduce(double (&v)[NV], double *partials,
                                            unsigned int *counter, F fin)
{
    __shared__ double sm[NV][kBlock / 32];
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
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double s = 0;
            for (int k = 0; k < nw; ++k) s += sm[i][k];
            t[i] = s;
        }
        fin(t);
        *counter = 0;
        __threadfence();
    }
}

__device__ __forceinline__ double round_to(double v, int single) { return single ? (double)(float)v : v; }

// true when the chunk-local iteration `gate` was cancelled by an earlier stop
__device__ __forceinline__ bool gated_off(const SolverState *st, int gate)
{
    return gate >= 0 && gate > *(volatile const int *)&st->stop_at;
}

inline int grid_for(int n) { return (n + kBlock - 1) / kBlock; }

}  // namespace qb
