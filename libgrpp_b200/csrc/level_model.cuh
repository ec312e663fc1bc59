// Learned grid-level model of the radial walk: a small MLP that predicts, from a
// task's angular momenta, geometry and exponents, the nested-grid level at which
// libgrpp's adaptive quadrature stops for that task (radial_type2_integral.c:285-315:
// the deepest level any entry of the task needs, 0..8).
//
// Network: 12 normalised features -> 64 -> 64 -> 64 (ReLU) -> 9 logits, argmax = level.
// Weights are used in BF16 with FP32 accumulation; training keeps FP32 master weights
// (Adam) and differentiates through the BF16-rounded weights (the values the forward
// pass used). Model layout (FP32, kLmParams floats):
//   mean[12] std[12] W1[64][12] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[9][64] b4[9]
//
// Kernels:
//   level_features_kernel  features of every radial item (one thread per item)
//   level_predict_kernel   MLP inference, one warp per item, BF16 weights in shared memory
//   level_order_kernel     deepest-predicted-first order of the items (counting sort)
//   mlp_train_kernel       forward + backward of a minibatch, 32 samples per CTA,
//                          gradients summed in shared memory and added to a global buffer
//   mlp_adam_kernel        Adam step on the master weights, BF16 copy for the next step
#pragma once

#include <cuda_bf16.h>

#include "grpp_common.cuh"
#include "radial.cuh"

namespace grpp {

constexpr int kLmFeat = 12, kLmHid = 64, kLmOut = 9;
constexpr int kLmOffMean = 0, kLmOffStd = kLmFeat;
constexpr int kLmOffW1 = 2 * kLmFeat;
constexpr int kLmOffB1 = kLmOffW1 + kLmHid * kLmFeat;
constexpr int kLmOffW2 = kLmOffB1 + kLmHid;
constexpr int kLmOffB2 = kLmOffW2 + kLmHid * kLmHid;
constexpr int kLmOffW3 = kLmOffB2 + kLmHid;
constexpr int kLmOffB3 = kLmOffW3 + kLmHid * kLmHid;
constexpr int kLmOffW4 = kLmOffB3 + kLmHid;
constexpr int kLmOffB4 = kLmOffW4 + kLmOut * kLmHid;
constexpr int kLmParams = kLmOffB4 + kLmOut;  // 9761
constexpr int kLmNet = kLmParams - kLmOffW1;   // trainable parameters (normalisation excluded)
constexpr int kLmTrainSamples = 32;            // samples per CTA in mlp_train_kernel
constexpr int kLmTrainThreads = 256;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// ---- features -------------------------------------------------------------------------
// la, lb, max projector L, number of semilocal potentials, log(1+|CA|), log(1+|CB|),
// log min/max exponent of A (radial-path primitives), of B, of the potential terms.
__device__ inline void item_features(const RadialArgs &a, int item, float *f)
{
    const int t = a.item_task[item];
    const int sa = a.task_a[t], sb = a.task_b[t], c = a.task_c[t];
    const double *Ao = a.shell_origin + 3 * sa, *Bo = a.shell_origin + 3 * sb, *Co = a.centre_origin + 3 * c;
    double CA2 = 0.0, CB2 = 0.0;
    for (int d = 0; d < 3; d++) {
        CA2 += (Co[d] - Ao[d]) * (Co[d] - Ao[d]);
        CB2 += (Co[d] - Bo[d]) * (Co[d] - Bo[d]);
    }
    const int g = a.centre_grpp[c], npot = a.grpp_sl_n[g], slo = a.grpp_sl_off[g];
    int Lmax = 0;
    double zmin = 1e300, zmax = 0.0;
    for (int p = 0; p < npot; p++) {
        const int pot = a.sl_pot[slo + p];
        Lmax = max(Lmax, a.pot_L[pot]);
        for (int k = 0; k < a.pot_nprim[pot]; k++) {
            const double z = a.pot_alpha[a.pot_prim_off[pot] + k];
            zmin = fmin(zmin, z);
            zmax = fmax(zmax, z);
        }
    }
    double amin = 1e300, amax = 0.0, bmin = 1e300, bmax = 0.0;
    for (int i = 0; i < a.rp_n[sa]; i++) {
        const double x = a.rp_alpha[a.rp_off[sa] + i];
        amin = fmin(amin, x);
        amax = fmax(amax, x);
    }
    for (int i = 0; i < a.rp_n[sb]; i++) {
        const double x = a.rp_alpha[a.rp_off[sb] + i];
        bmin = fmin(bmin, x);
        bmax = fmax(bmax, x);
    }
    auto lg = [](double x) { return (float)log(fmax(x, 1e-30)); };
    f[0] = (float)a.shell_L[sa];
    f[1] = (float)a.shell_L[sb];
    f[2] = (float)Lmax;
    f[3] = (float)npot;
    f[4] = (float)log1p(sqrt(CA2));
    f[5] = (float)log1p(sqrt(CB2));
    f[6] = lg(amin);
    f[7] = lg(amax);
    f[8] = lg(bmin);
    f[9] = lg(bmax);
    f[10] = lg(zmin);
    f[11] = lg(zmax);
}

__global__ void level_features_kernel(RadialArgs a, float *feat)
{
    for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < a.n_items; item += gridDim.x * blockDim.x)
        item_features(a, item, feat + (size_t)item * kLmFeat);
}

// ---- inference ----------------------------------------------------------------------------
// One warp per item; lane j owns hidden units j and j + 32. The normalisation is kept
// in FP32; the weights are BF16 (same layout as the parameter vector, first 24 unused).
struct LevelModelDev {
    const float *norm;          // mean[12], std[12] (FP32)
    const __nv_bfloat16 *w;     // kLmParams BF16 values (same layout; the first 24 unused)
};

__device__ inline int mlp_forward_warp(const LevelModelDev &m, const float *x_raw, float *hbuf, int lane)
{
    // hbuf: 2 x 64 floats private to the warp
    float *ha = hbuf, *hb = hbuf + kLmHid;
    if (lane < kLmFeat) ha[lane] = (x_raw[lane] - m.norm[lane]) / m.norm[kLmFeat + lane];
    __syncwarp();
    float out[2];
    for (int q = 0; q < 2; q++) {
        const int j = lane + 32 * q;
        float s = __bfloat162float(m.w[kLmOffB1 + j]);
        for (int k = 0; k < kLmFeat; k++) s += __bfloat162float(m.w[kLmOffW1 + j * kLmFeat + k]) * ha[k];
        out[q] = fmaxf(s, 0.f);
    }
    __syncwarp();
    hb[lane] = out[0];
    hb[lane + 32] = out[1];
    __syncwarp();
    const int offW[2] = {kLmOffW2, kLmOffW3}, offB[2] = {kLmOffB2, kLmOffB3};
    float *src = hb, *dst = ha;
    for (int layer = 0; layer < 2; layer++) {
        for (int q = 0; q < 2; q++) {
            const int j = lane + 32 * q;
            float s = __bfloat162float(m.w[offB[layer] + j]);
            for (int k = 0; k < kLmHid; k++) s += __bfloat162float(m.w[offW[layer] + j * kLmHid + k]) * src[k];
            out[q] = fmaxf(s, 0.f);
        }
        __syncwarp();
        dst[lane] = out[0];
        dst[lane + 32] = out[1];
        __syncwarp();
        float *tmp = src;
        src = dst;
        dst = tmp;
    }
    float logit = -INFINITY;
    if (lane < kLmOut) {
        float s = __bfloat162float(m.w[kLmOffB4 + lane]);
        for (int k = 0; k < kLmHid; k++) s += __bfloat162float(m.w[kLmOffW4 + lane * kLmHid + k]) * src[k];
        logit = s;
    }
    // argmax over the 9 logits (lowest level on ties)
    int best = lane < kLmOut ? lane : kLmOut;
    float bv = logit;
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, best, o);
        if (ov > bv || (ov == bv && oi < best)) {
            bv = ov;
            best = oi;
        }
    }
    __syncwarp();
    return best;
}

// pred[item] = predicted level of walked items, -1 for items without grid work
__global__ void __launch_bounds__(128) level_predict_kernel(RadialArgs a, LevelModelDev m, int8_t *pred)
{
    __shared__ float hbuf[4][2 * kLmHid];
    __shared__ float xbuf[4][kLmFeat];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int item = blockIdx.x * 4 + warp; item < a.n_items; item += gridDim.x * 4) {
        if (!a.walk[item]) {
            if (lane == 0) pred[item] = -1;
            continue;
        }
        if (lane == 0) item_features(a, item, xbuf[warp]);
        __syncwarp();
        const int lvl = mlp_forward_warp(m, xbuf[warp], hbuf[warp], lane);
        if (lane == 0) pred[item] = (int8_t)lvl;
        __syncwarp();
    }
}

// Deepest-predicted-first order of the walked items: counting sort over levels 8..0.
// cursor[0..9] must be zero on entry; one CTA of 256 threads.
__global__ void level_order_kernel(int n_items, const int8_t *pred, int *order, int *n_order, int *cursor)
{
    __shared__ int hist[kLmOut], start[kLmOut];
    if (threadIdx.x < kLmOut) hist[threadIdx.x] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n_items; i += blockDim.x)
        if (pred[i] >= 0) atomicAdd(&hist[min((int)pred[i], kLmOut - 1)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int l = kLmOut - 1; l >= 0; l--) {
            start[l] = s;
            s += hist[l];
        }
        *n_order = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_items; i += blockDim.x)
        if (pred[i] >= 0) {
            const int l = min((int)pred[i], kLmOut - 1);
            order[start[l] + atomicAdd(&cursor[l], 1)] = i;
        }
}

// ---- training -----------------------------------------------------------------------------
struct MlpTrainArgs {
    const float *X;             // [n][12] raw features
    const int8_t *y;            // [n] levels 0..8
    const int *idx;             // [n] sample order of this epoch
    int n, b0, bsz;             // samples b0 .. b0+bsz-1 of the order form the minibatch
    const float *norm;          // mean, std
    const __nv_bfloat16 *w;     // BF16 weights used by the forward pass (kLmParams, first 24 unused)
    float *grad;                // kLmParams (first 24 unused), summed over the minibatch, / bsz
    float *loss;                // summed cross-entropy / bsz
};

// shared layout (floats): W [kLmParams] | G [kLmParams] | x [S][12] | h1 h2 h3 [S][64] | d [S][64] | e [S][64] | p [S][9]
constexpr size_t mlp_train_smem_bytes()
{
    return sizeof(float) * (2 * (size_t)kLmParams + kLmTrainSamples * (kLmFeat + 5 * kLmHid + kLmOut));
}

__global__ void __launch_bounds__(kLmTrainThreads) mlp_train_kernel(MlpTrainArgs t)
{
    extern __shared__ float sm[];
    float *W = sm, *G = W + kLmParams, *x = G + kLmParams;
    float *h1 = x + kLmTrainSamples * kLmFeat, *h2 = h1 + kLmTrainSamples * kLmHid, *h3 = h2 + kLmTrainSamples * kLmHid;
    float *d = h3 + kLmTrainSamples * kLmHid, *e = d + kLmTrainSamples * kLmHid, *p = e + kLmTrainSamples * kLmHid;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int s0 = blockIdx.x * kLmTrainSamples;
    const int ns = min(kLmTrainSamples, t.bsz - s0);
    if (ns <= 0) return;
    for (int i = tid; i < kLmParams; i += nt) {
        W[i] = i < kLmOffW1 ? 0.f : __bfloat162float(t.w[i]);
        G[i] = 0.f;
    }
    for (int i = tid; i < kLmTrainSamples * kLmFeat; i += nt) {
        const int s = i / kLmFeat, k = i % kLmFeat;
        float v = 0.f;
        if (s < ns) {
            const int smp = t.idx[t.b0 + s0 + s];
            v = (t.X[(size_t)smp * kLmFeat + k] - t.norm[k]) / t.norm[kLmFeat + k];
        }
        x[i] = v;
    }
    __syncthreads();
    // forward: h1 = relu(W1 x + b1), h2, h3, logits
    auto dense = [&](const float *in, int nin, int woff, int boff, int nout, float *out, bool relu) {
        for (int i = tid; i < kLmTrainSamples * nout; i += nt) {
            const int s = i / nout, j = i % nout;
            float acc = W[boff + j];
            for (int k = 0; k < nin; k++) acc += W[woff + j * nin + k] * in[s * nin + k];
            out[i] = relu ? fmaxf(acc, 0.f) : acc;
        }
        __syncthreads();
    };
    dense(x, kLmFeat, kLmOffW1, kLmOffB1, kLmHid, h1, true);
    dense(h1, kLmHid, kLmOffW2, kLmOffB2, kLmHid, h2, true);
    dense(h2, kLmHid, kLmOffW3, kLmOffB3, kLmHid, h3, true);
    dense(h3, kLmHid, kLmOffW4, kLmOffB4, kLmOut, p, false);
    // softmax cross-entropy; p <- dL/dlogits = (softmax - onehot) / bsz
    const float inv_b = 1.f / (float)t.bsz;
    if (tid < kLmTrainSamples) {
        const int s = tid;
        float l = 0.f;
        if (s < ns) {
            float mx = -INFINITY;
            for (int c = 0; c < kLmOut; c++) mx = fmaxf(mx, p[s * kLmOut + c]);
            float z = 0.f;
            for (int c = 0; c < kLmOut; c++) z += expf(p[s * kLmOut + c] - mx);
            const int y = t.y[t.idx[t.b0 + s0 + s]];
            l = -(p[s * kLmOut + y] - mx - logf(z));
            for (int c = 0; c < kLmOut; c++)
                p[s * kLmOut + c] = (expf(p[s * kLmOut + c] - mx) / z - (c == y ? 1.f : 0.f)) * inv_b;
        } else {
            for (int c = 0; c < kLmOut; c++) p[s * kLmOut + c] = 0.f;
        }
        for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
        if (tid == 0) atomicAdd(t.loss, l * inv_b);
    }
    __syncthreads();
    // backward of one dense layer: dW += dout^T in, db += sum dout, din = (W^T dout) * relu'(in)
    auto back = [&](const float *dout, int nout, const float *in, int nin, int woff, int boff, float *din) {
        for (int i = tid; i < nout * nin; i += nt) {
            const int j = i / nin, k = i % nin;
            float acc = 0.f;
            for (int s = 0; s < kLmTrainSamples; s++) acc += dout[s * nout + j] * in[s * nin + k];
            G[woff + i] += acc;
        }
        for (int j = tid; j < nout; j += nt) {
            float acc = 0.f;
            for (int s = 0; s < kLmTrainSamples; s++) acc += dout[s * nout + j];
            G[boff + j] += acc;
        }
        if (din) {
            for (int i = tid; i < kLmTrainSamples * nin; i += nt) {
                const int s = i / nin, k = i % nin;
                float acc = 0.f;
                for (int j = 0; j < nout; j++) acc += W[woff + j * nin + k] * dout[s * nout + j];
                din[i] = in[i] > 0.f ? acc : 0.f;
            }
        }
        __syncthreads();
    };
    back(p, kLmOut, h3, kLmHid, kLmOffW4, kLmOffB4, d);
    back(d, kLmHid, h2, kLmHid, kLmOffW3, kLmOffB3, e);
    back(e, kLmHid, h1, kLmHid, kLmOffW2, kLmOffB2, d);
    back(d, kLmHid, x, kLmFeat, kLmOffW1, kLmOffB1, nullptr);
    for (int i = kLmOffW1 + tid; i < kLmParams; i += nt) atomicAdd(t.grad + i, G[i]);
}

struct AdamArgs {
    float *w;                   // FP32 master weights (kLmParams)
    __nv_bfloat16 *wb;          // BF16 copy used by the forward pass
    float *grad, *m, *v;        // gradient (zeroed after the step), moments
    float lr, beta1, beta2, eps, bc1, bc2;  // bc = 1 - beta^t
};

__global__ void mlp_adam_kernel(AdamArgs a)
{
    for (int i = kLmOffW1 + blockIdx.x * blockDim.x + threadIdx.x; i < kLmParams; i += gridDim.x * blockDim.x) {
        const float g = a.grad[i];
        const float m = a.beta1 * a.m[i] + (1.f - a.beta1) * g;
        const float v = a.beta2 * a.v[i] + (1.f - a.beta2) * g * g;
        a.m[i] = m;
        a.v[i] = v;
        const float w = a.w[i] - a.lr * (m / a.bc1) / (sqrtf(v / a.bc2) + a.eps);
        a.w[i] = w;
        a.wb[i] = __float2bfloat16_rn(w);
        a.grad[i] = 0.f;
    }
}

__global__ void mlp_to_bf16_kernel(const float *w, __nv_bfloat16 *wb, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) wb[i] = __float2bfloat16_rn(w[i]);
}

}  // namespace grpp
