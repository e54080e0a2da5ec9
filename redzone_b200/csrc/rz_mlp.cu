// rz_mlp.cu -- learned launch-configuration predictor: features, FP32 MLP training and inference.
//
// The network maps 12 features of a removal instance to 63 logits (softmax over the launch
// configurations of config_space(), rz_autotune.cpp) plus one logit for "the O(n) partition
// path beats Redzone". Layers: 12 -> 64 (ReLU) -> 64 (ReLU) -> 64. All arithmetic is FP32 in
// hand-written kernels (no cuBLAS): one warp per sample for the forward and backward passes
// with the weights staged in shared memory, one thread per parameter for the weight gradients
// and the Adam update. Training targets are the kernels' own timings (soft targets favouring
// configurations within a few percent of the fastest); see redzone_b200/learn.py.
//
// Features (rz_mlp_features), computed on the GPU from the index list itself:
//   0 log2(n)/32   1 log2(k)/32   2 k/n   3 payload bytes/32
//   4, 5  mean and variance of log2(1 + gap / (n/S)) over the sorted sample of S <= 4096 indices
//   6     fraction of the sample in the red zone [n-k, n)
//   7-11  run-length histogram of the sorted sample (runs of consecutive indices of length
//         1, 2-3, 4-15, 16-63, >= 64), as fractions of the runs
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "rz_common.cuh"
#include "rz_internal.h"

namespace rz {

constexpr int kIn = 12, kH = 64, kCfg = kConfigSpace, kOut = kCfg + 1;
static_assert(kCfg >= 32 && kOut <= 64, "one warp holds the logits two per lane");
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kIn * kH;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kH * kOut;
constexpr int kParams = kOffB3 + kOut;  // 9152
constexpr int kSample = 4096;
constexpr float kBitWeight = 0.5f;  // weight of the partition-bit loss

// ---- features -----------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) features_kernel(const uint32_t* __restrict__ idx, uint32_t n, uint32_t k,
                                                        uint32_t w, float* __restrict__ out) {
    __shared__ uint32_t s[kSample];
    __shared__ float red[2][32];
    __shared__ uint32_t hist[5];
    __shared__ uint32_t s_runs, s_tail;
    const int tid = threadIdx.x, B = blockDim.x;
    const uint32_t S = min(k, uint32_t(kSample));
    for (int i = tid; i < kSample; i += B) s[i] = (uint32_t(i) < S) ? __ldg(&idx[i]) : 0xffffffffu;
    if (tid < 5) hist[tid] = 0;
    if (tid == 0) {
        s_runs = 0;
        s_tail = 0;
    }
    __syncthreads();
    // Bitonic sort of the 4096-entry sample (padding sorts to the end).
    for (int size = 2; size <= kSample; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = tid; i < kSample; i += B) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = ((i & size) == 0);
                    const uint32_t a = s[i], b = s[j];
                    if ((a > b) == up) {
                        s[i] = b;
                        s[j] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    const float scale = float(n) / float(max(S, 1u));
    const uint32_t cut = n - k;
    float sum = 0.f, sum2 = 0.f;
    for (uint32_t i = tid; i < S; i += B) {
        if (s[i] >= cut) atomicAdd(&s_tail, 1u);
        if (i + 1 < S) {
            const float x = log2f(1.f + float(s[i + 1] - s[i]) / scale);
            sum += x;
            sum2 += x * x;
        }
        // Run starts: first element or not adjacent to the previous one.
        if (i == 0 || s[i] != s[i - 1] + 1u) {
            uint32_t len = 1;
            while (i + len < S && s[i + len] == s[i + len - 1] + 1u) ++len;
            const int b = len == 1 ? 0 : len < 4 ? 1 : len < 16 ? 2 : len < 64 ? 3 : 4;
            atomicAdd(&hist[b], 1u);
            atomicAdd(&s_runs, 1u);
        }
    }
    for (int d = 16; d > 0; d >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, d);
        sum2 += __shfl_down_sync(0xffffffffu, sum2, d);
    }
    if ((tid & 31) == 0) {
        red[0][tid >> 5] = sum;
        red[1][tid >> 5] = sum2;
    }
    __syncthreads();
    if (tid == 0) {
        float a = 0.f, b = 0.f;
        for (int q = 0; q < B / 32; ++q) {
            a += red[0][q];
            b += red[1][q];
        }
        const float m = S > 1 ? a / float(S - 1) : 0.f;
        const float v = S > 1 ? fmaxf(b / float(S - 1) - m * m, 0.f) : 0.f;
        out[0] = log2f(float(max(n, 1u))) / 32.f;
        out[1] = log2f(float(max(k, 1u))) / 32.f;
        out[2] = float(k) / float(max(n, 1u));
        out[3] = float(w) / 32.f;
        out[4] = m / 8.f;
        out[5] = v / 16.f;
        out[6] = S ? float(s_tail) / float(S) : 0.f;
        const float runs = float(max(s_runs, 1u));
        for (int q = 0; q < 5; ++q) out[7 + q] = float(hist[q]) / runs;
    }
}

// ---- forward (+ loss gradient) ------------------------------------------------------------------
// One warp per sample: lane l owns hidden units l and l+32 and outputs l, l+32 (< kOut).
__global__ void __launch_bounds__(256) mlp_forward_kernel(const float* __restrict__ P, const float* __restrict__ X,
                                                          const float* __restrict__ Tg, const int* __restrict__ order,
                                                          int nsamp, float* __restrict__ H1, float* __restrict__ H2,
                                                          float* __restrict__ O, float* __restrict__ dO,
                                                          float* __restrict__ loss) {
    __shared__ float sp[kParams];
    __shared__ float sh[8][2 * kH];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) sp[i] = P[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const int b = blockIdx.x * (blockDim.x >> 5) + wq;
    if (b >= nsamp) return;
    const int src = order ? order[b] : b;
    const float* x = X + size_t(src) * kIn;
    float xin[kIn];
#pragma unroll
    for (int i = 0; i < kIn; ++i) xin[i] = __ldg(&x[i]);
    float* h1 = sh[wq];
    float* h2 = sh[wq] + kH;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int u = lane + 32 * r;
        float a = sp[kOffB1 + u];
#pragma unroll
        for (int i = 0; i < kIn; ++i) a += xin[i] * sp[kOffW1 + i * kH + u];
        h1[u] = fmaxf(a, 0.f);
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int u = lane + 32 * r;
        float a = sp[kOffB2 + u];
        for (int i = 0; i < kH; ++i) a += h1[i] * sp[kOffW2 + i * kH + u];
        h2[u] = fmaxf(a, 0.f);
    }
    __syncwarp();
    float o[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int u = lane + 32 * r;
        float a = 0.f;
        if (u < kOut) {
            a = sp[kOffB3 + u];
            for (int i = 0; i < kH; ++i) a += h2[i] * sp[kOffW3 + i * kOut + u];
        }
        o[r] = a;
    }
    if (H1) {
        H1[size_t(b) * kH + lane] = h1[lane];
        H1[size_t(b) * kH + lane + 32] = h1[lane + 32];
        H2[size_t(b) * kH + lane] = h2[lane];
        H2[size_t(b) * kH + lane + 32] = h2[lane + 32];
    }
    O[size_t(b) * kOut + lane] = o[0];
    if (lane + 32 < kOut) O[size_t(b) * kOut + lane + 32] = o[1];
    if (!Tg) return;
    // Softmax cross-entropy over the kCfg configuration logits (soft targets) + weighted binary
    // cross-entropy of the partition bit (logit kCfg). Gradients are averaged over the batch.
    const float* t = Tg + size_t(src) * kOut;
    const float l0 = o[0];                                        // unit lane (< kCfg always)
    const float l1 = (lane + 32 < kCfg) ? o[1] : -INFINITY;       // units 32..kCfg-1
    float mx = fmaxf(l0, l1);
    for (int d = 16; d > 0; d >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, d));
    const float e0 = __expf(l0 - mx), e1 = (lane + 32 < kCfg) ? __expf(l1 - mx) : 0.f;
    float se = e0 + e1;
    for (int d = 16; d > 0; d >>= 1) se += __shfl_xor_sync(0xffffffffu, se, d);
    const float lse = mx + __logf(se);
    const float t0 = __ldg(&t[lane]);
    const float t1 = (lane + 32 < kCfg) ? __ldg(&t[lane + 32]) : 0.f;
    float ce = -(t0 * (l0 - lse)) - ((lane + 32 < kCfg) ? t1 * (l1 - lse) : 0.f);
    for (int d = 16; d > 0; d >>= 1) ce += __shfl_xor_sync(0xffffffffu, ce, d);
    const float inv = 1.f / float(nsamp);
    dO[size_t(b) * kOut + lane] = (e0 / se - t0) * inv;
    if (lane + 32 < kCfg) dO[size_t(b) * kOut + lane + 32] = (e1 / se - t1) * inv;
    if (lane == kCfg - 32) {  // unit kCfg: the partition bit
        const float z = o[1];
        const float tb = __ldg(&t[kCfg]);
        const float pz = 1.f / (1.f + __expf(-z));
        dO[size_t(b) * kOut + kCfg] = kBitWeight * (pz - tb) * inv;
        const float bce = fmaxf(z, 0.f) - z * tb + __logf(1.f + __expf(-fabsf(z)));
        atomicAdd(loss, (ce + kBitWeight * bce) * inv);
    }
}

// ---- backward through the hidden layers ---------------------------------------------------------
__global__ void __launch_bounds__(256) mlp_backward_kernel(const float* __restrict__ P, const float* __restrict__ H1,
                                                           const float* __restrict__ H2, const float* __restrict__ dO,
                                                           int nsamp, float* __restrict__ dH1,
                                                           float* __restrict__ dH2) {
    __shared__ float sp[kParams];
    __shared__ float sd[8][kOut + kH];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) sp[i] = P[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const int b = blockIdx.x * (blockDim.x >> 5) + wq;
    if (b >= nsamp) return;
    float* go = sd[wq];
    float* g2 = sd[wq] + kOut;
    go[lane] = dO[size_t(b) * kOut + lane];
    if (lane + 32 < kOut) go[lane + 32] = dO[size_t(b) * kOut + lane + 32];
    __syncwarp();
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int u = lane + 32 * r;
        float a = 0.f;
        for (int j = 0; j < kOut; ++j) a += go[j] * sp[kOffW3 + u * kOut + j];
        a = H2[size_t(b) * kH + u] > 0.f ? a : 0.f;
        g2[u] = a;
        dH2[size_t(b) * kH + u] = a;
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int u = lane + 32 * r;
        float a = 0.f;
        for (int j = 0; j < kH; ++j) a += g2[j] * sp[kOffW2 + u * kH + j];
        dH1[size_t(b) * kH + u] = H1[size_t(b) * kH + u] > 0.f ? a : 0.f;
    }
}

// ---- weight gradients: one thread per parameter, summed over the batch ---------------------------
__global__ void mlp_weight_grad_kernel(const float* __restrict__ X, const int* __restrict__ order,
                                       const float* __restrict__ H1, const float* __restrict__ H2,
                                       const float* __restrict__ dH1, const float* __restrict__ dH2,
                                       const float* __restrict__ dO, int nsamp, float* __restrict__ G) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kParams) return;
    float acc = 0.f;
    if (q < kOffB1) {
        const int i = q / kH, j = q % kH;
        for (int b = 0; b < nsamp; ++b) acc += X[size_t(order ? order[b] : b) * kIn + i] * dH1[size_t(b) * kH + j];
    } else if (q < kOffW2) {
        const int j = q - kOffB1;
        for (int b = 0; b < nsamp; ++b) acc += dH1[size_t(b) * kH + j];
    } else if (q < kOffB2) {
        const int i = (q - kOffW2) / kH, j = (q - kOffW2) % kH;
        for (int b = 0; b < nsamp; ++b) acc += H1[size_t(b) * kH + i] * dH2[size_t(b) * kH + j];
    } else if (q < kOffW3) {
        const int j = q - kOffB2;
        for (int b = 0; b < nsamp; ++b) acc += dH2[size_t(b) * kH + j];
    } else if (q < kOffB3) {
        const int i = (q - kOffW3) / kOut, j = (q - kOffW3) % kOut;
        for (int b = 0; b < nsamp; ++b) acc += H2[size_t(b) * kH + i] * dO[size_t(b) * kOut + j];
    } else {
        const int j = q - kOffB3;
        for (int b = 0; b < nsamp; ++b) acc += dO[size_t(b) * kOut + j];
    }
    G[q] = acc;
}

// ---- Adam ---------------------------------------------------------------------------------------
__global__ void adam_kernel(float* __restrict__ P, float* __restrict__ M, float* __restrict__ V,
                            const float* __restrict__ G, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kParams) return;
    const float g = G[q];
    const float m = b1 * M[q] + (1.f - b1) * g;
    const float v = b2 * V[q] + (1.f - b2) * g * g;
    M[q] = m;
    V[q] = v;
    P[q] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

// ------------------------------------------------------------------------------------------------
struct Predictor;

}  // namespace rz

struct rz_mlp {
    rz_ctx* ctx = nullptr;
    float* P = nullptr;   // parameters (kParams)
    float* M = nullptr;   // Adam first moments
    float* V = nullptr;   // Adam second moments
    float* G = nullptr;   // gradient
    float* scratch = nullptr;  // per-batch activations
    size_t scratch_cap = 0;    // samples the activation scratch holds
    float* loss = nullptr;
    int step = 0;
};

namespace rz {

struct Predictor {
    rz_mlp* mlp = nullptr;        // single lists: launch configuration + partition bit
    rz_mlp* batch_mlp = nullptr;  // list mixes: batched configuration (outputs 0..kBatchCfgSpace-1)
    float* d_feat = nullptr;  // 12 floats
    float* d_out = nullptr;   // kOut floats
};

static int ensure_batch(rz_mlp* m, size_t nsamp) {
    if (nsamp <= m->scratch_cap) return RZ_OK;
    if (m->scratch) cudaFree(m->scratch);
    m->scratch = nullptr;
    const size_t per = size_t(2 * kH + kOut + kOut + 2 * kH);  // H1 H2 O dO dH1 dH2
    RZ_CUDA_TRY(m->ctx, cudaMalloc(&m->scratch, per * nsamp * sizeof(float)));
    m->scratch_cap = nsamp;
    return RZ_OK;
}

struct BatchBufs {
    float *H1, *H2, *O, *dO, *dH1, *dH2;
};
static BatchBufs bufs(rz_mlp* m, size_t cap) {
    BatchBufs b;
    b.H1 = m->scratch;
    b.H2 = b.H1 + cap * kH;
    b.O = b.H2 + cap * kH;
    b.dO = b.O + cap * kOut;
    b.dH1 = b.dO + cap * kOut;
    b.dH2 = b.dH1 + cap * kH;
    return b;
}

// One training step (or gradient evaluation) over `nsamp` samples selected by d_order.
static int run_step(rz_mlp* m, const float* dX, const float* dT, const int* d_order, int nsamp, bool update, float lr,
                    cudaStream_t s) {
    int st = ensure_batch(m, size_t(nsamp));
    if (st != RZ_OK) return st;
    BatchBufs b = bufs(m, m->scratch_cap);
    const int wpb = 8;
    const int grid = (nsamp + wpb - 1) / wpb;
    RZ_CUDA_TRY(m->ctx, cudaMemsetAsync(m->loss, 0, sizeof(float), s));
    mlp_forward_kernel<<<grid, 256, 0, s>>>(m->P, dX, dT, d_order, nsamp, b.H1, b.H2, b.O, b.dO, m->loss);
    mlp_backward_kernel<<<grid, 256, 0, s>>>(m->P, b.H1, b.H2, b.dO, nsamp, b.dH1, b.dH2);
    mlp_weight_grad_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(dX, d_order, b.H1, b.H2, b.dH1, b.dH2, b.dO, nsamp,
                                                                 m->G);
    if (update) {
        ++m->step;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, float(m->step)), c2 = 1.f - std::pow(b2, float(m->step));
        adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(m->P, m->M, m->V, m->G, lr, b1, b2, 1e-8f, c1, c2);
    }
    RZ_CUDA_TRY(m->ctx, cudaGetLastError());
    return RZ_OK;
}

bool predict_cfg(rz_ctx* ctx, uint32_t n, uint32_t k, uint32_t w, const uint32_t* d_idx, cudaStream_t s,
                 rz_launch_cfg* cfg) {
    Predictor* pr = static_cast<Predictor*>(ctx->predictor);
    if (!pr || !pr->mlp || k == 0) return false;
    features_kernel<<<1, 1024, 0, s>>>(d_idx, n, k, w, pr->d_feat);
    mlp_forward_kernel<<<1, 32, 0, s>>>(pr->mlp->P, pr->d_feat, nullptr, nullptr, 1, nullptr, nullptr, pr->d_out,
                                        nullptr, nullptr);
    float o[kOut];
    if (cudaMemcpyAsync(o, pr->d_out, sizeof(o), cudaMemcpyDeviceToHost, s) != cudaSuccess) return false;
    if (cudaStreamSynchronize(s) != cudaSuccess) return false;
    int best = 0;
    for (int q = 1; q < kCfg; ++q)
        if (o[q] > o[best]) best = q;
    rz_launch_cfg space[kCfg];
    config_space(space);
    *cfg = space[best];
    cfg->use_partition = o[kCfg] > 0.f ? 1 : 0;
    return true;
}

// ---- list mixes (the batched kernel) -----------------------------------------------------------
// The same network, trained separately, maps 12 features of a mix of lists to logits over the
// batched configuration space (outputs 0..kBatchCfgSpace-1; the others are trained towards zero
// probability and ignored). Features, computed on the host from the list sizes alone, each scaled
// to about [0, 1]:
//   0 log2(lists)/16   1 log2(1 + total n)/36   2 log2(1 + total k)/36   3 total k / total n
//   4 payload bytes/32   5, 6 mean and standard deviation of log2(1 + n) over the lists (/32, /8)
//   7 mean of k/n over the lists
//   8-10 share of the removals in lists with k <= 256, <= 1024, <= 4096 (lists that one CTA
//        removes whole with the smaller tiles)   11 log2(1 + largest k)/24
void batch_config_space(rz_batch_cfg* out) {
    int q = 0;
    for (int b : {128, 256, 512})
        for (int i : {2, 4, 8})
            for (int c : {1, 2, 4})
                for (int wave : {0, kDefaultWave}) out[q++] = rz_batch_cfg{b, i, c, 0, wave};
}

void batch_features(const rz_list_desc* lists, int nlists, uint32_t w, float* f) {
    double tn = 0, tk = 0, mlog = 0, mlog2 = 0, mf = 0, s256 = 0, s1k = 0, s4k = 0, kmax = 0;
    int used = 0;
    for (int l = 0; l < nlists; ++l) {
        const double n = double(lists[l].n), k = double(lists[l].k);
        if (n <= 0) continue;
        ++used;
        tn += n;
        tk += k;
        const double lg = std::log2(1.0 + n);
        mlog += lg;
        mlog2 += lg * lg;
        mf += k / n;
        if (k <= 256) s256 += k;
        if (k <= 1024) s1k += k;
        if (k <= 4096) s4k += k;
        kmax = std::max(kmax, k);
    }
    const double u = std::max(used, 1);
    mlog /= u;
    const double var = std::max(0.0, mlog2 / u - mlog * mlog);
    f[0] = float(std::log2(std::max(1.0, double(nlists))) / 16.0);
    f[1] = float(std::log2(1.0 + tn) / 36.0);
    f[2] = float(std::log2(1.0 + tk) / 36.0);
    f[3] = float(tn > 0 ? tk / tn : 0.0);
    f[4] = float(w) / 32.f;
    f[5] = float(mlog / 32.0);
    f[6] = float(std::sqrt(var) / 8.0);
    f[7] = float(mf / u);
    f[8] = float(tk > 0 ? s256 / tk : 0.0);
    f[9] = float(tk > 0 ? s1k / tk : 0.0);
    f[10] = float(tk > 0 ? s4k / tk : 0.0);
    f[11] = float(std::log2(1.0 + kmax) / 24.0);
}

bool predict_batch_cfg(rz_ctx* ctx, const rz_list_desc* lists, int nlists, uint32_t w, rz_batch_cfg* cfg) {
    Predictor* pr = static_cast<Predictor*>(ctx->predictor);
    if (!pr || !pr->batch_mlp || nlists < 1) return false;
    float feat[kIn];
    batch_features(lists, nlists, w, feat);
    if (cudaMemcpy(pr->d_feat, feat, sizeof(feat), cudaMemcpyHostToDevice) != cudaSuccess) return false;
    mlp_forward_kernel<<<1, 32>>>(pr->batch_mlp->P, pr->d_feat, nullptr, nullptr, 1, nullptr, nullptr, pr->d_out,
                                  nullptr, nullptr);
    float o[kOut];
    if (cudaMemcpy(o, pr->d_out, sizeof(o), cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    // Only configurations whose tile lets the longest list fit in the batched kernel's tile limit
    // are candidates (the others cannot plan this mix).
    int64_t kmax = 0;
    for (int l = 0; l < nlists; ++l)
        if (lists[l].k < lists[l].n) kmax = std::max<int64_t>(kmax, lists[l].k);
    rz_batch_cfg space[kBatchCfgSpace];
    batch_config_space(space);
    int best = -1;
    for (int q = 0; q < kBatchCfgSpace; ++q) {
        if (int64_t(space[q].block) * space[q].items * kBatchMaxTilesPerList < kmax) continue;
        if (best < 0 || o[q] > o[best]) best = q;
    }
    if (best < 0) return false;
    *cfg = space[best];
    return true;
}

void release_predictor(rz_ctx* ctx) {
    Predictor* pr = static_cast<Predictor*>(ctx->predictor);
    if (!pr) return;
    cudaFree(pr->d_feat);
    delete pr;
    ctx->predictor = nullptr;
}

}  // namespace rz

using namespace rz;

extern "C" {

int rz_mlp_param_count(void) { return kParams; }

int rz_mlp_create(rz_ctx* ctx, uint64_t seed, rz_mlp** out) {
    if (!ctx || !out) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    rz_mlp* m = new (std::nothrow) rz_mlp();
    if (!m) return RZ_ERR_NO_MEMORY;
    m->ctx = ctx;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, (4 * size_t(kParams) + 1) * sizeof(float));
    if (e != cudaSuccess) {
        delete m;
        return cuda_fail(ctx, e, "rz_mlp_create");
    }
    m->P = static_cast<float*>(p);
    m->M = m->P + kParams;
    m->V = m->M + kParams;
    m->G = m->V + kParams;
    m->loss = m->G + kParams;
    // He-uniform initialisation from a seeded generator; biases zero.
    std::vector<float> h(kParams, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_in, int count) {
        const float lim = std::sqrt(6.f / float(fan_in));
        std::uniform_real_distribution<float> u(-lim, lim);
        for (int i = 0; i < count; ++i) h[size_t(off + i)] = u(rng);
    };
    fill(kOffW1, kIn, kIn * kH);
    fill(kOffW2, kH, kH * kH);
    fill(kOffW3, kH, kH * kOut);
    e = cudaMemcpy(m->P, h.data(), kParams * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->M, 0, 2 * kParams * sizeof(float));
    if (e != cudaSuccess) {
        cudaFree(m->P);
        delete m;
        return cuda_fail(ctx, e, "rz_mlp_create");
    }
    *out = m;
    return RZ_OK;
}

void rz_mlp_destroy(rz_mlp* m) {
    if (!m) return;
    cudaSetDevice(m->ctx->device);
    Predictor* pr = static_cast<Predictor*>(m->ctx->predictor);
    if (pr && pr->mlp == m) pr->mlp = nullptr;
    if (pr && pr->batch_mlp == m) pr->batch_mlp = nullptr;
    cudaFree(m->P);
    cudaFree(m->scratch);
    delete m;
}

int rz_mlp_get_params(rz_mlp* m, float* h_params, int32_t count) {
    if (!m || !h_params || count != kParams) return RZ_ERR_INVALID_ARG;
    RZ_CUDA_TRY(m->ctx, cudaMemcpy(h_params, m->P, kParams * sizeof(float), cudaMemcpyDeviceToHost));
    return RZ_OK;
}

int rz_mlp_set_params(rz_mlp* m, const float* h_params, int32_t count) {
    if (!m || !h_params || count != kParams) return RZ_ERR_INVALID_ARG;
    RZ_CUDA_TRY(m->ctx, cudaMemcpy(m->P, h_params, kParams * sizeof(float), cudaMemcpyHostToDevice));
    RZ_CUDA_TRY(m->ctx, cudaMemset(m->M, 0, 2 * kParams * sizeof(float)));
    m->step = 0;
    return RZ_OK;
}

int rz_mlp_features(rz_ctx* ctx, const uint32_t* d_idx, int64_t n, int64_t k, uint32_t elem_bytes, float* h_feat12) {
    if (!ctx || !h_feat12 || n < 0 || k < 0 || k > n || n >= (int64_t(1) << 32) || (k > 0 && !d_idx))
        return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    float* d = nullptr;
    RZ_CUDA_TRY(ctx, cudaMalloc(&d, kIn * sizeof(float)));
    features_kernel<<<1, 1024>>>(d_idx, uint32_t(n), uint32_t(k), elem_bytes, d);
    cudaError_t e = cudaMemcpy(h_feat12, d, kIn * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "rz_mlp_features");
    return RZ_OK;
}

// Forward pass over host features (nsamp x 12) -> host logits (nsamp x kOut).
int rz_mlp_forward(rz_mlp* m, const float* h_x, int64_t nsamp, float* h_out) {
    if (!m || !h_x || !h_out || nsamp < 1) return RZ_ERR_INVALID_ARG;
    rz_ctx* ctx = m->ctx;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    float *dx = nullptr, *dout = nullptr;
    RZ_CUDA_TRY(ctx, cudaMalloc(&dx, size_t(nsamp) * (kIn + kOut) * sizeof(float)));
    dout = dx + size_t(nsamp) * kIn;
    cudaError_t e = cudaMemcpy(dx, h_x, size_t(nsamp) * kIn * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        mlp_forward_kernel<<<int((nsamp + 7) / 8), 256>>>(m->P, dx, nullptr, nullptr, int(nsamp), nullptr, nullptr,
                                                          dout, nullptr, nullptr);
        e = cudaMemcpy(h_out, dout, size_t(nsamp) * kOut * sizeof(float), cudaMemcpyDeviceToHost);
    }
    cudaFree(dx);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "rz_mlp_forward");
    return RZ_OK;
}

// Mean loss and the gradient of every parameter over one batch (host in, host out).
int rz_mlp_gradients(rz_mlp* m, const float* h_x, const float* h_t, int64_t nsamp, float* h_grad, float* h_loss) {
    if (!m || !h_x || !h_t || !h_grad || nsamp < 1 || nsamp > 65536) return RZ_ERR_INVALID_ARG;
    rz_ctx* ctx = m->ctx;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    float* d = nullptr;
    RZ_CUDA_TRY(ctx, cudaMalloc(&d, size_t(nsamp) * (kIn + kOut) * sizeof(float)));
    cudaError_t e = cudaMemcpy(d, h_x, size_t(nsamp) * kIn * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d + size_t(nsamp) * kIn, h_t, size_t(nsamp) * kOut * sizeof(float), cudaMemcpyHostToDevice);
    int st = (e == cudaSuccess) ? run_step(m, d, d + size_t(nsamp) * kIn, nullptr, int(nsamp), false, 0.f, nullptr)
                                : cuda_fail(ctx, e, "rz_mlp_gradients");
    if (st == RZ_OK) {
        e = cudaMemcpy(h_grad, m->G, kParams * sizeof(float), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && h_loss) e = cudaMemcpy(h_loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = cuda_fail(ctx, e, "rz_mlp_gradients");
    }
    cudaFree(d);
    return st;
}

// Adam training on the GPU: nsamp samples (12 features, kOut targets each), mini-batches drawn by a
// seeded shuffle every epoch. *h_last_loss receives the mean loss of the last epoch.
int rz_mlp_train(rz_mlp* m, const float* h_x, const float* h_t, int64_t nsamp, int32_t epochs, int32_t batch,
                 float lr, uint64_t seed, float* h_last_loss) {
    if (!m || !h_x || !h_t || nsamp < 1 || epochs < 1 || batch < 1 || batch > 65536) return RZ_ERR_INVALID_ARG;
    rz_ctx* ctx = m->ctx;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    float* d = nullptr;
    int* dord = nullptr;
    RZ_CUDA_TRY(ctx, cudaMalloc(&d, size_t(nsamp) * (kIn + kOut) * sizeof(float)));
    cudaError_t e = cudaMalloc(&dord, size_t(nsamp) * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(d, h_x, size_t(nsamp) * kIn * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d + size_t(nsamp) * kIn, h_t, size_t(nsamp) * kOut * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        cudaFree(dord);
        return cuda_fail(ctx, e, "rz_mlp_train upload");
    }
    std::vector<int> order(static_cast<size_t>(nsamp));
    for (int64_t i = 0; i < nsamp; ++i) order[size_t(i)] = int(i);
    std::mt19937_64 rng(seed);
    int st = RZ_OK;
    double epoch_loss = 0.0;
    for (int ep = 0; ep < epochs && st == RZ_OK; ++ep) {
        std::shuffle(order.begin(), order.end(), rng);
        e = cudaMemcpy(dord, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            st = cuda_fail(ctx, e, "rz_mlp_train order");
            break;
        }
        epoch_loss = 0.0;
        int nb = 0;
        for (int64_t b0 = 0; b0 < nsamp && st == RZ_OK; b0 += batch) {
            const int nbatch = int(std::min<int64_t>(batch, nsamp - b0));
            st = run_step(m, d, d + size_t(nsamp) * kIn, dord + b0, nbatch, true, lr, nullptr);
            if (ep == epochs - 1 && st == RZ_OK) {
                float l = 0.f;
                cudaMemcpy(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost);
                epoch_loss += l;
                ++nb;
            }
        }
        if (nb) epoch_loss /= nb;
    }
    cudaDeviceSynchronize();
    cudaFree(d);
    cudaFree(dord);
    if (h_last_loss) *h_last_loss = float(epoch_loss);
    return st;
}

static int ensure_predictor(rz_ctx* ctx, Predictor** out) {
    Predictor* pr = static_cast<Predictor*>(ctx->predictor);
    if (!pr) {
        pr = new (std::nothrow) Predictor();
        if (!pr) return RZ_ERR_NO_MEMORY;
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, (kIn + kOut) * sizeof(float));
        if (e != cudaSuccess) {
            delete pr;
            return cuda_fail(ctx, e, "predictor");
        }
        pr->d_feat = static_cast<float*>(p);
        pr->d_out = pr->d_feat + kIn;
        ctx->predictor = pr;
    }
    *out = pr;
    return RZ_OK;
}

int rz_set_predictor(rz_ctx* ctx, rz_mlp* m) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    Predictor* pr = nullptr;
    const int st = ensure_predictor(ctx, &pr);
    if (st != RZ_OK) return st;
    pr->mlp = m;
    return RZ_OK;
}

int rz_set_batch_predictor(rz_ctx* ctx, rz_mlp* m) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    Predictor* pr = nullptr;
    const int st = ensure_predictor(ctx, &pr);
    if (st != RZ_OK) return st;
    pr->batch_mlp = m;
    return RZ_OK;
}

int rz_batch_config_space(rz_batch_cfg* out, int32_t max) {
    rz_batch_cfg space[kBatchCfgSpace];
    batch_config_space(space);
    if (out)
        for (int q = 0; q < std::min<int>(max, kBatchCfgSpace); ++q) out[q] = space[q];
    return kBatchCfgSpace;
}

int rz_batch_features(const rz_list_desc* lists, int32_t nlists, uint32_t elem_bytes, float* h_features12) {
    if (!h_features12 || nlists < 0 || (nlists > 0 && !lists)) return RZ_ERR_INVALID_ARG;
    batch_features(lists, nlists, elem_bytes, h_features12);
    return RZ_OK;
}

int rz_predict_batch_cfg(rz_ctx* ctx, const rz_list_desc* lists, int32_t nlists, uint32_t elem_bytes,
                         rz_batch_cfg* cfg) {
    if (!ctx || !cfg || nlists < 0 || (nlists > 0 && !lists)) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return predict_batch_cfg(ctx, lists, nlists, elem_bytes, cfg) ? RZ_OK : RZ_ERR_UNSUPPORTED;
}

int rz_predict_cfg(rz_ctx* ctx, const uint32_t* d_idx, int64_t n, int64_t k, uint32_t elem_bytes, rz_launch_cfg* cfg) {
    if (!ctx || !cfg || k < 0 || k > n || n >= (int64_t(1) << 32)) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return predict_cfg(ctx, uint32_t(n), uint32_t(k), elem_bytes, d_idx, nullptr, cfg) ? RZ_OK : RZ_ERR_UNSUPPORTED;
}

}  // extern "C"
