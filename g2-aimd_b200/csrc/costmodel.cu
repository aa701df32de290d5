// costmodel.cu - the learned root-cost model: features, training, inference.
//
// A root task's cost (SM cycles of its search, logged by the enumeration
// kernels) is predicted by an MLP 8 -> 64 -> 64 -> 1 (ReLU) from 8 per-root
// features.  Weights are kept as fp32 masters and used as bf16 operands of
// tensor-core MMAs (mma.sync m16n8k16, fp32 accumulate); training is one fused
// forward+backward kernel per mini-batch plus an Adam update kernel.  The model
// only orders and splits root tasks; it never touches the enumeration results.
//
// Features of root v (ids in degeneracy order), all log1p-scaled except f6:
//   f0 deg(v)           f1 core(v)            f2 p = |N+(v)|        f3 |N-(v)|
//   f4 sum_{u in N+(v)} |N+(u)| (forward wedge count)
//   f5 mean, f7 max of |N+(v) ∩ N+(u)| over up to 4 sampled u in N+(v)
//   f6 that mean divided by p (sampled local density)
// Inputs to the MLP are (f - mean) / std with the training set's statistics;
// the output is the normalised log1p(cost).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "g2_device.cuh"
#include "g2_kernels.h"

namespace g2 {

namespace {

constexpr int F = 8, KP = 16, H = 64;  // features, padded K of layer 1, hidden width

struct ModelView {  // offsets into the flat fp32 parameter vector (G2_MODEL_PARAMS)
    static constexpr int W1 = 0;             // [H][F]
    static constexpr int B1 = W1 + H * F;    // [H]
    static constexpr int W2 = B1 + H;        // [H][H]
    static constexpr int B2 = W2 + H * H;    // [H]
    static constexpr int W3 = B2 + H;        // [H]
    static constexpr int B3 = W3 + H;        // [1]
    static constexpr int N = B3 + 1;
};
static_assert(ModelView::N == G2_MODEL_PARAMS, "parameter layout");

// ------------------------------------------------------------ features

__device__ void root_features(const uint64_t *rp, const uint32_t *ci, const uint32_t *fo, const uint32_t *core,
                              uint32_t v, float *f) {
    const uint64_t lo = rp[v], hi = rp[v + 1];
    const uint64_t s = lo + fo[v];
    const uint32_t p = (uint32_t)(hi - s), nx = (uint32_t)(s - lo);
    float wedge = 0.f, isum = 0.f, imax = 0.f;
    for (uint32_t i = 0; i < p; i++) {
        const uint32_t u = ci[s + i];
        wedge += (float)(rp[u + 1] - rp[u] - fo[u]);
    }
    const uint32_t ns = p < 4 ? p : 4;
    for (uint32_t j = 0; j < ns; j++) {
        const uint32_t u = ci[s + (uint64_t)j * p / ns];
        const uint64_t us = rp[u] + fo[u], ue = rp[u + 1];
        uint32_t c = 0;
        uint64_t pos = s;
        for (uint64_t e = us; e < ue; e++) {  // |N+(u) ∩ N+(v)|, both sorted
            const uint32_t y = ci[e];
            pos = lower_bound(ci, pos, hi, y);
            if (pos >= hi) break;
            c += ci[pos] == y;
        }
        isum += (float)c;
        imax = (float)c > imax ? (float)c : imax;
    }
    const float imean = ns ? isum / (float)ns : 0.f;
    f[0] = log1pf((float)(hi - lo));
    f[1] = log1pf((float)(core ? core[v] : p));
    f[2] = log1pf((float)p);
    f[3] = log1pf((float)nx);
    f[4] = log1pf(wedge);
    f[5] = log1pf(imean);
    f[6] = p ? imean / (float)p : 0.f;
    f[7] = log1pf(imax);
}

// One warp per root: lanes share the wedge sum and each sampled intersection
// (integer sums, so the result equals root_features() exactly).
__global__ void features_kernel(const uint64_t *rp, const uint32_t *ci, const uint32_t *fo, const uint32_t *core,
                                const uint32_t *src, uint64_t n, float *out) {
    const uint32_t lane = lane_id();
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = warp; i < n; i += nwarps) {
        const uint32_t v = src ? src[i] : (uint32_t)i;
        const uint64_t lo = rp[v], hi = rp[v + 1];
        const uint64_t s = lo + fo[v];
        const uint32_t p = (uint32_t)(hi - s), nx = (uint32_t)(s - lo);
        unsigned long long wedge = 0;
        for (uint32_t j = lane; j < p; j += 32) {
            const uint32_t u = ci[s + j];
            wedge += rp[u + 1] - rp[u] - fo[u];
        }
        wedge = warp_sum_u64(wedge);
        const uint32_t ns = p < 4 ? p : 4;
        const uint32_t pmax = p ? ci[hi - 1] : 0u;
        uint32_t isum = 0, imax = 0;
        for (uint32_t j = 0; j < ns; j++) {
            const uint32_t u = ci[s + (uint64_t)j * p / ns];
            const uint64_t us = rp[u] + fo[u], ue = rp[u + 1];
            uint32_t c = 0;
            for (uint64_t e = us + lane; e < ue; e += 32) {  // |N+(u) ∩ N+(v)|
                const uint32_t y = ci[e];
                if (y > pmax) break;
                c += contains(ci, s, hi, y);
            }
            c = (uint32_t)warp_sum_u64(c);
            isum += c;
            imax = c > imax ? c : imax;
        }
        if (lane == 0) {
            const float imean = ns ? (float)isum / (float)ns : 0.f;
            float *f = out + i * F;
            f[0] = log1pf((float)(hi - lo));
            f[1] = log1pf((float)(core ? core[v] : p));
            f[2] = log1pf((float)p);
            f[3] = log1pf((float)nx);
            f[4] = log1pf((float)wedge);
            f[5] = log1pf(imean);
            f[6] = p ? imean / (float)p : 0.f;
            f[7] = log1pf((float)imax);
        }
    }
}

// ------------------------------------------------- tensor-core MMA helpers

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 t = __floats2bfloat162_rn(lo, hi);  // .x = lo (low half), .y = hi
    return *reinterpret_cast<uint32_t *>(&t);
}

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16(x)); }

// D = A(16x16, row) * B(16x8, col) + C, bf16 inputs, fp32 accumulate.
__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Fragment loads with explicit element indexing (operand layouts of the PTX ISA
// for m16n8k16: g = lane / 4, t = lane % 4; C element (g or g+8, 2t or 2t+1)).
// A(m, k) and B(k, n) are read through accessors, so transposed operands need
// no data movement.
template <class FA>
__device__ __forceinline__ void load_a(uint32_t a[4], FA A) {
    const int g = lane_id() >> 2, t = lane_id() & 3;
    a[0] = pack_bf16(A(g, 2 * t), A(g, 2 * t + 1));
    a[1] = pack_bf16(A(g + 8, 2 * t), A(g + 8, 2 * t + 1));
    a[2] = pack_bf16(A(g, 2 * t + 8), A(g, 2 * t + 9));
    a[3] = pack_bf16(A(g + 8, 2 * t + 8), A(g + 8, 2 * t + 9));
}
template <class FB>
__device__ __forceinline__ void load_b(uint32_t b[2], FB B) {
    const int g = lane_id() >> 2, t = lane_id() & 3;
    b[0] = pack_bf16(B(2 * t, g), B(2 * t + 1, g));
    b[1] = pack_bf16(B(2 * t + 8, g), B(2 * t + 9, g));
}

// Per-warp shared staging for 16 rows.
struct WarpTile {
    float x[16][KP];   // normalised inputs (zero padded to 16)
    float h1[16][H];   // post-ReLU layer-1 activations
    float h2[16][H];   // post-ReLU layer-2 activations
    float d2[16][H];   // dL/d(pre-activation 2)
    float d1[16][H];   // dL/d(pre-activation 1)
    float y[16];
};

// Model weights (fp32) staged per CTA in shared memory.
struct SharedModel {
    float w1[H][KP];
    float b1[H];
    float w2[H][H];
    float b2[H];
    float w3[H];
    float b3;
    float mean[F], stdinv[F];
};

__device__ void stage_model(SharedModel &m, const float *params, const float *norm) {
    for (int i = threadIdx.x; i < H * KP; i += blockDim.x) {
        const int r = i / KP, c = i % KP;
        m.w1[r][c] = c < F ? params[ModelView::W1 + r * F + c] : 0.f;
    }
    for (int i = threadIdx.x; i < H * H; i += blockDim.x) m.w2[i / H][i % H] = params[ModelView::W2 + i];
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        m.b1[i] = params[ModelView::B1 + i];
        m.b2[i] = params[ModelView::B2 + i];
        m.w3[i] = params[ModelView::W3 + i];
    }
    if (threadIdx.x == 0) m.b3 = params[ModelView::B3];
    for (int i = threadIdx.x; i < F; i += blockDim.x) {
        m.mean[i] = norm[i];
        m.stdinv[i] = 1.f / norm[F + i];
    }
    __syncthreads();
}

// Forward of the 16 rows held in t.x: fills t.h1, t.h2, t.y (whole warp).
__device__ void forward16(const SharedModel &m, WarpTile &t) {
    const int g = lane_id() >> 2, q = lane_id() & 3;
    uint32_t ax[4];
    load_a(ax, [&](int r, int c) { return t.x[r][c]; });
    // layer 1: [16 x 16] x [16 x 64]
    for (int nt = 0; nt < H / 8; nt++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        uint32_t b[2];
        load_b(b, [&](int k, int n) { return m.w1[nt * 8 + n][k]; });
        mma16816(c, ax, b);
        const int col = nt * 8 + 2 * q;
        t.h1[g][col] = fmaxf(c[0] + m.b1[col], 0.f);
        t.h1[g][col + 1] = fmaxf(c[1] + m.b1[col + 1], 0.f);
        t.h1[g + 8][col] = fmaxf(c[2] + m.b1[col], 0.f);
        t.h1[g + 8][col + 1] = fmaxf(c[3] + m.b1[col + 1], 0.f);
    }
    __syncwarp();
    // layer 2: [16 x 64] x [64 x 64]
    uint32_t ah[4][4];
    for (int kt = 0; kt < H / 16; kt++) load_a(ah[kt], [&](int r, int c) { return t.h1[r][kt * 16 + c]; });
    for (int nt = 0; nt < H / 8; nt++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        for (int kt = 0; kt < H / 16; kt++) {
            uint32_t b[2];
            load_b(b, [&](int k, int n) { return m.w2[nt * 8 + n][kt * 16 + k]; });
            mma16816(c, ah[kt], b);
        }
        const int col = nt * 8 + 2 * q;
        t.h2[g][col] = fmaxf(c[0] + m.b2[col], 0.f);
        t.h2[g][col + 1] = fmaxf(c[1] + m.b2[col + 1], 0.f);
        t.h2[g + 8][col] = fmaxf(c[2] + m.b2[col], 0.f);
        t.h2[g + 8][col + 1] = fmaxf(c[3] + m.b2[col + 1], 0.f);
    }
    __syncwarp();
    // layer 3 (64 -> 1) on the CUDA cores with bf16-rounded operands
    if (lane_id() < 16) {
        const int r = lane_id();
        float s = m.b3;
        for (int k = 0; k < H; k++) s += bf16r(t.h2[r][k]) * bf16r(m.w3[k]);
        t.y[r] = s;
    }
    __syncwarp();
}

__device__ void normalise_row(const SharedModel &m, const float *f, float *x) {
    for (int k = 0; k < F; k++) x[k] = (f[k] - m.mean[k]) * m.stdinv[k];
    for (int k = F; k < KP; k++) x[k] = 0.f;
}

// ------------------------------------------------------------- training

// One mini-batch of n rows (ids idx[0..n) into X / Y): forward, squared error
// against the normalised targets Y, backward; gradients of the MEAN squared
// error accumulated into grad (fp32 atomics), the summed squared error into
// loss.  4 warps x 16 rows per CTA.
__global__ void __launch_bounds__(128) train_step_kernel(const float *X, const float *Y, const uint32_t *idx,
                                                         uint32_t n, const float *params, const float *norm,
                                                         float *grad, float *loss, float inv_batch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SharedModel &m = *reinterpret_cast<SharedModel *>(smem_raw);
    WarpTile *tiles = reinterpret_cast<WarpTile *>(smem_raw + sizeof(SharedModel));
    stage_model(m, params, norm);
    const int w = threadIdx.x >> 5, lane = lane_id();
    WarpTile &t = tiles[w];
    const uint32_t row0 = (blockIdx.x * 4 + w) * 16;
    if (row0 >= n) return;  // warp-uniform; no CTA barrier follows
    const int g = lane >> 2, q = lane & 3;
    // inputs of 16 rows (rows past n are zero and carry no loss)
    if (lane < 16) {
        const uint32_t r = row0 + lane;
        if (r < n) {
            float f[F];
            for (int k = 0; k < F; k++) f[k] = X[(uint64_t)idx[r] * F + k];
            normalise_row(m, f, t.x[lane]);
        } else {
            for (int k = 0; k < KP; k++) t.x[lane][k] = 0.f;
        }
    }
    __syncwarp();
    forward16(m, t);
    // dL/dy (lane r holds row r) and the loss
    float dy = 0.f;
    if (lane < 16) {
        const uint32_t r = row0 + lane;
        if (r < n) {
            const float e = t.y[lane] - Y[idx[r]];
            atomicAdd(loss, e * e);
            dy = 2.f * e * inv_batch;
        }
    }
    // head: dw3 = sum_r dy_r h2_r, db3 = sum_r dy_r
    for (int k = lane; k < H; k += 32) {
        float s = 0.f;
        for (int r = 0; r < 16; r++) s += __shfl_sync(G2_FULL, dy, r) * t.h2[r][k];
        atomicAdd(grad + ModelView::W3 + k, s);
    }
    {
        float s = 0.f;
        for (int r = 0; r < 16; r++) s += __shfl_sync(G2_FULL, dy, r);
        if (lane == 0) atomicAdd(grad + ModelView::B3, s);
    }
    // d2[r][k] = dy_r * w3[k] * relu'(h2[r][k])
    for (int r = 0; r < 16; r++) {
        const float dyr = __shfl_sync(G2_FULL, dy, r);
        for (int k = lane; k < H; k += 32) t.d2[r][k] = t.h2[r][k] > 0.f ? dyr * bf16r(m.w3[k]) : 0.f;
    }
    __syncwarp();
    // dW2 (64 x 64) = d2^T (64 out x 16 rows) x h1 (16 rows x 64 in)
    for (int mt = 0; mt < H / 16; mt++) {
        uint32_t a[4];
        load_a(a, [&](int mm, int kk) { return t.d2[kk][mt * 16 + mm]; });
        for (int nt = 0; nt < H / 8; nt++) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            uint32_t b[2];
            load_b(b, [&](int kk, int nn) { return t.h1[kk][nt * 8 + nn]; });
            mma16816(c, a, b);
            const int o = mt * 16 + g, i = nt * 8 + 2 * q;
            atomicAdd(grad + ModelView::W2 + o * H + i, c[0]);
            atomicAdd(grad + ModelView::W2 + o * H + i + 1, c[1]);
            atomicAdd(grad + ModelView::W2 + (o + 8) * H + i, c[2]);
            atomicAdd(grad + ModelView::W2 + (o + 8) * H + i + 1, c[3]);
        }
    }
    for (int k = lane; k < H; k += 32) {
        float s = 0.f;
        for (int r = 0; r < 16; r++) s += t.d2[r][k];
        atomicAdd(grad + ModelView::B2 + k, s);
    }
    // d1 (16 x 64 in) = d2 (16 x 64 out) x W2 (64 out x 64 in), masked by relu'(h1)
    {
        uint32_t ad[4][4];
        for (int kt = 0; kt < H / 16; kt++) load_a(ad[kt], [&](int r, int c) { return t.d2[r][kt * 16 + c]; });
        for (int nt = 0; nt < H / 8; nt++) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            for (int kt = 0; kt < H / 16; kt++) {
                uint32_t b[2];
                load_b(b, [&](int kk, int nn) { return m.w2[kt * 16 + kk][nt * 8 + nn]; });
                mma16816(c, ad[kt], b);
            }
            const int col = nt * 8 + 2 * q;
            t.d1[g][col] = t.h1[g][col] > 0.f ? c[0] : 0.f;
            t.d1[g][col + 1] = t.h1[g][col + 1] > 0.f ? c[1] : 0.f;
            t.d1[g + 8][col] = t.h1[g + 8][col] > 0.f ? c[2] : 0.f;
            t.d1[g + 8][col + 1] = t.h1[g + 8][col + 1] > 0.f ? c[3] : 0.f;
        }
    }
    __syncwarp();
    // dW1 (64 x 8) = d1^T (64 x 16 rows) x x (16 rows x 16 padded in)
    for (int mt = 0; mt < H / 16; mt++) {
        uint32_t a[4];
        load_a(a, [&](int mm, int kk) { return t.d1[kk][mt * 16 + mm]; });
        for (int nt = 0; nt < KP / 8; nt++) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            uint32_t b[2];
            load_b(b, [&](int kk, int nn) { return t.x[kk][nt * 8 + nn]; });
            mma16816(c, a, b);
            const int o = mt * 16 + g, i = nt * 8 + 2 * q;
            if (i < F) {
                atomicAdd(grad + ModelView::W1 + o * F + i, c[0]);
                atomicAdd(grad + ModelView::W1 + (o + 8) * F + i, c[2]);
            }
            if (i + 1 < F) {
                atomicAdd(grad + ModelView::W1 + o * F + i + 1, c[1]);
                atomicAdd(grad + ModelView::W1 + (o + 8) * F + i + 1, c[3]);
            }
        }
    }
    for (int k = lane; k < H; k += 32) {
        float s = 0.f;
        for (int r = 0; r < 16; r++) s += t.d1[r][k];
        atomicAdd(grad + ModelView::B1 + k, s);
    }
}

__global__ void adam_kernel(float *params, float *mom, float *vel, const float *grad, int n, float lr, float b1t,
                            float b2t) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = grad[i];
        const float mi = b1 * mom[i] + (1.f - b1) * gi;
        const float vi = b2 * vel[i] + (1.f - b2) * gi * gi;
        mom[i] = mi;
        vel[i] = vi;
        params[i] -= lr * (mi / (1.f - b1t)) / (sqrtf(vi / (1.f - b2t)) + eps);
    }
}

// ------------------------------------------------------------- inference

// Features + MLP of every root in one kernel (the inference fused into task
// generation).  pred[i] (optional) = normalised log-cost of root src[i];
// cost[i] (optional) = decoded cost (>= 1); *total (optional) += sum of costs.
// With X given, the features are read from X instead: row src[i] (per-vertex
// features cached for the loaded graph) or row i when src is null.
__global__ void __launch_bounds__(128) score_kernel(const uint64_t *rp, const uint32_t *ci, const uint32_t *fo,
                                                    const uint32_t *core, const uint32_t *src, uint64_t n,
                                                    const float *X, const float *params, const float *norm,
                                                    float *pred, float *cost, float *total) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SharedModel &m = *reinterpret_cast<SharedModel *>(smem_raw);
    WarpTile *tiles = reinterpret_cast<WarpTile *>(smem_raw + sizeof(SharedModel));
    stage_model(m, params, norm);
    const int w = threadIdx.x >> 5, lane = lane_id();
    WarpTile &t = tiles[w];
    const float ymean = norm[2 * F], ystd = norm[2 * F + 1];
    float local = 0.f;
    for (uint64_t base = ((uint64_t)blockIdx.x * 4 + w) * 16; base < n; base += (uint64_t)gridDim.x * 4 * 16) {
        if (lane < 16) {
            const uint64_t i = base + lane;
            if (i < n) {
                float f[F];
                if (X) {  // precomputed features, rows indexed by vertex when src is given
                    const uint64_t row = src ? (uint64_t)src[i] : i;
                    for (int k = 0; k < F; k++) f[k] = X[row * F + k];
                }
                else
                    root_features(rp, ci, fo, core, src ? src[i] : (uint32_t)i, f);
                normalise_row(m, f, t.x[lane]);
            } else {
                for (int k = 0; k < KP; k++) t.x[lane][k] = 0.f;
            }
        }
        __syncwarp();
        forward16(m, t);
        if (lane < 16) {
            const uint64_t i = base + lane;
            if (i < n) {
                const float y = t.y[lane];
                const float c = expm1f(fminf(y * ystd + ymean, 80.f));  // targets are log1p(cycles)
                const float cc = c > 1.f ? c : 1.f;
                if (pred) pred[i] = y;
                if (cost) cost[i] = cc;
                local += cc;
            }
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(G2_FULL, local, o);
    if (lane == 0 && total) atomicAdd(total, local);
}

}  // namespace

size_t model_smem_bytes() { return sizeof(SharedModel) + 4 * sizeof(WarpTile); }

cudaError_t features_launch(const uint64_t *rp, const uint32_t *ci, const uint32_t *fo, const uint32_t *core,
                            const uint32_t *src, uint64_t n, float *out, int sms, cudaStream_t st) {
    features_kernel<<<sms * 16, 256, 0, st>>>(rp, ci, fo, core, src, n, out);
    return cudaGetLastError();
}

cudaError_t train_step_launch(const float *X, const float *Y, const uint32_t *idx, uint32_t n, const float *params,
                              const float *norm, float *grad, float *loss, cudaStream_t st) {
    const size_t sm = model_smem_bytes();
    cudaFuncSetAttribute(train_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    const uint32_t blocks = (n + 63) / 64;
    train_step_kernel<<<blocks, 128, sm, st>>>(X, Y, idx, n, params, norm, grad, loss, 1.f / (float)n);
    return cudaGetLastError();
}

cudaError_t adam_launch(float *params, float *mom, float *vel, const float *grad, float lr, int step,
                        cudaStream_t st) {
    const float b1t = powf(0.9f, (float)step), b2t = powf(0.999f, (float)step);
    adam_kernel<<<(G2_MODEL_PARAMS + 255) / 256, 256, 0, st>>>(params, mom, vel, grad, G2_MODEL_PARAMS, lr, b1t, b2t);
    return cudaGetLastError();
}

cudaError_t score_launch(const uint64_t *rp, const uint32_t *ci, const uint32_t *fo, const uint32_t *core,
                         const uint32_t *src, uint64_t n, const float *X, const float *params, const float *norm,
                         float *pred, float *cost, float *total, int sms, cudaStream_t st) {
    const size_t sm = model_smem_bytes();
    cudaFuncSetAttribute(score_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    score_kernel<<<sms * 4, 128, sm, st>>>(rp, ci, fo, core, src, n, X, params, norm, pred, cost, total);
    return cudaGetLastError();
}

}  // namespace g2
