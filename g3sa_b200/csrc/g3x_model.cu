// g3x_model.cu -- learned per-job cost model: features, an MLP 5 -> 64 -> 64 -> 1 (ReLU,
// fp32, 4,609 parameters), and its forward, backward and Adam kernels.
//
// The model predicts a job's work (the caller trains it on log2(1 + DP cells) measured by
// the extension kernel's own cell counters) from five features of the job header and its
// sequences.  The scheduler orders and buckets jobs by the prediction; scores never depend
// on it.
//
// Parameter layout (floats): W1[64][5] | b1[64] | W2[64][64] | b2[64] | W3[64] | b3.
// Training works on one mini-batch at a time as a sequence of small kernels; every gradient
// is a fixed-order sum over the batch (no atomics), so training is deterministic.
#include <cuda_runtime.h>
#include <math.h>
#include "g3x_internal.h"
#include "g3x_stage.cuh"
#include "g3x_schedkey.cuh"

namespace g3x {

constexpr int kF = 5, kH = 64;
constexpr int oW1 = 0, ob1 = oW1 + kH * kF, oW2 = ob1 + kH, ob2 = oW2 + kH * kH, oW3 = ob2 + kH,
              ob3 = oW3 + kH, kParams = ob3 + 1;
static_assert(oW2 % 4 == 0 && kH % 4 == 0, "W2 rows load as float4");
static_assert(kParams == G3X_MLP_PARAMS, "parameter count");

// ---- features ---------------------------------------------------------------------------

// Per job: qlen/128, tlen/256, h0/64, and the ungapped extension along the seed's diagonal
// over the first min(qlen, tlen) bases (from h0, +1 per identical base pair, -4 per other pair):
// its best score / 64 and the bases at which that score is first reached / 128.  Where the
// diagonal's score peaks tells how far the alignment runs before z-drop, and how high, how wide
// its band grows.
// The first three 16-base chunks of a job's query and target as load16 leaves them (2-bit codes,
// N bits), and which of them are loaded.
struct Head48 {
    uint32_t qx[3], qn[3], tx[3], tn[3];
    int loaded;                          // chunks 0 .. loaded - 1 of both sequences
};

// head (optional) keeps the chunks the diagonal walk loads among the first three.
__device__ __forceinline__ void job_features(const g3x_job_t& jb, const uint32_t* __restrict__ codes,
                                             const uint32_t* __restrict__ nmask, int64_t n_bases,
                                             float (&f)[kF], Head48* head = nullptr) {
    const bool qrev = (jb.flags & G3X_JOB_QREV) != 0, trev = (jb.flags & G3X_JOB_TREV) != 0;
    // (a job reaching past the planes reads nothing: its diagonal stays at h0)
    const int kk = !job_in_planes(jb, n_bases) ? 0 : (jb.qlen < jb.tlen ? jb.qlen : jb.tlen);
    int32_t sc = jb.h0, best = jb.h0, best_at = 0;
    for (int ch = 0; (ch << 4) < kk; ++ch) {
        uint32_t xq, nq, xt, nt;
        load16(codes, nmask, jb.q_off, jb.qlen, ch, qrev, xq, nq);
        load16(codes, nmask, jb.t_off, jb.tlen, ch, trev, xt, nt);
        if (head && ch < 3) {                      // (constant indices: the chunks stay in registers)
#pragma unroll
            for (int c3 = 0; c3 < 3; ++c3)
                if (c3 == ch) { head->qx[c3] = xq; head->qn[c3] = nq; head->tx[c3] = xt; head->tn[c3] = nt; }
            head->loaded = ch + 1;
        }
        const int nv = kk - (ch << 4) < 16 ? kk - (ch << 4) : 16;
        // bit t of m: base t of the chunk differs (2-bit codes differ, or N on either side)
        const uint32_t d2 = xq ^ xt;
        uint32_t m = (d2 | (d2 >> 1)) & 0x55555555u;
        m = (m | (m >> 1)) & 0x33333333u;
        m = (m | (m >> 2)) & 0x0F0F0F0Fu;
        m = (m | (m >> 4)) & 0x00FF00FFu;
        m = ((m | (m >> 8)) | nq | nt) & 0xFFFFu;
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            if (t < nv) {
                sc += 1 - 5 * (int32_t)((m >> t) & 1u);
                const bool up = sc > best;
                best = up ? sc : best;
                best_at = up ? (ch << 4) + t + 1 : best_at;
            }
        }
    }
    f[0] = jb.qlen * (1.0f / 128.0f);
    f[1] = jb.tlen * (1.0f / 256.0f);
    f[2] = jb.h0 * (1.0f / 64.0f);
    f[3] = best * (1.0f / 64.0f);
    f[4] = best_at * (1.0f / 128.0f);
}

// Whether one of the 16 diagonals next to the seed's (offsets 1-8 either way) matches at least
// kNearMatch of its first kNearLen base pairs (N on either side is no match).  The learned
// schedule asks this of the jobs the network calls early-ending: such a job's seed is followed
// by an indel and then by the same sequence, which its ungapped features (the seed's own
// diagonal) cannot see, and it runs most of its rows; on config-2 jobs the check holds for about
// 60% of the network's false early calls and for almost none of its right ones.
constexpr int kNearDiag = 8, kNearLen = 32, kNearMatch = 18;

// Bases 0 .. 47 of one sequence as 2-bit codes (lo: bases 0-31, hi: 32-47) and N bits, from the
// chunks the feature walk loaded (the first `have`) and the planes for the rest.
__device__ __forceinline__ void load48(const uint32_t* __restrict__ codes, const uint32_t* __restrict__ nmask,
                                       uint32_t off, int len, bool rev, const uint32_t (&hx)[3],
                                       const uint32_t (&hn)[3], int have, uint64_t& lo, uint32_t& hi,
                                       uint64_t& nb) {
    uint32_t x[3] = {0u, 0u, 0u}, n[3] = {0u, 0u, 0u};
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        if (ch < have) { x[ch] = hx[ch]; n[ch] = hn[ch]; }
        else if ((ch << 4) < len) load16(codes, nmask, off, len, ch, rev, x[ch], n[ch]);
    }
    lo = (uint64_t)x[0] | ((uint64_t)x[1] << 32);
    hi = x[2];
    nb = (uint64_t)n[0] | ((uint64_t)n[1] << 16) | ((uint64_t)n[2] << 32);
}

// 32 bases from base a (0 <= a <= 8) of a sequence held as load48 leaves it.
__device__ __forceinline__ uint64_t window32(uint64_t lo, uint32_t hi, int a) {
    return a == 0 ? lo : (lo >> (2 * a)) | ((uint64_t)hi << (64 - 2 * a));
}

__device__ bool near_diagonal(const g3x_job_t& jb, const uint32_t* __restrict__ codes,
                              const uint32_t* __restrict__ nmask, int64_t n_bases, const Head48& head) {
    if (!job_in_planes(jb, n_bases)) return false;
    uint64_t qlo, tlo, qn, tn;
    uint32_t qhi, thi;
    load48(codes, nmask, jb.q_off, jb.qlen, (jb.flags & G3X_JOB_QREV) != 0, head.qx, head.qn, head.loaded,
           qlo, qhi, qn);
    load48(codes, nmask, jb.t_off, jb.tlen, (jb.flags & G3X_JOB_TREV) != 0, head.tx, head.tn, head.loaded,
           tlo, thi, tn);
#pragma unroll 1
    for (int s = 0; s < 2 * kNearDiag; ++s) {
        // offsets 1..8: query base k against target base k + d; -1..-8: query k + d, target k
        const int d = 1 + (s >> 1), a = (s & 1) ? d : 0, b = (s & 1) ? 0 : d;
        const int kk = min(kNearLen, min(jb.qlen - a, jb.tlen - b));
        if (kk < kNearMatch) continue;
        uint64_t x = window32(qlo, qhi, a) ^ window32(tlo, thi, b);
        x = (x | (x >> 1)) & 0x5555555555555555ull;            // one bit per base: codes differ
        x = (x | (x >> 1)) & 0x3333333333333333ull;
        x = (x | (x >> 2)) & 0x0F0F0F0F0F0F0F0Full;
        x = (x | (x >> 4)) & 0x00FF00FF00FF00FFull;
        x = (x | (x >> 8)) & 0x0000FFFF0000FFFFull;
        const uint32_t diff = (uint32_t)(x | (x >> 16)) | (uint32_t)(qn >> a) | (uint32_t)(tn >> b);
        const uint32_t valid = kk >= 32 ? 0xFFFFFFFFu : (1u << kk) - 1u;
        if (__popc(~diff & valid) >= kNearMatch) return true;
    }
    return false;
}

// One thread per job.
__global__ void features_kernel(const g3x_job_t* __restrict__ jobs, int n,
                                const uint32_t* __restrict__ codes,
                                const uint32_t* __restrict__ nmask, int64_t n_bases, float* __restrict__ feat,
                                const int32_t* __restrict__ subset, const int32_t* __restrict__ subset_n) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || (subset_n && k >= *subset_n)) return;
    if (subset) k = subset[k];              // features of job subset[k], stored at that job
    float f[kF];
    job_features(jobs[k], codes, nmask, n_bases, f);
    float* o = feat + (size_t)k * kF;
#pragma unroll
    for (int i = 0; i < kF; ++i) o[i] = f[i];
}

// ---- inference ---------------------------------------------------------------------------

// Two jobs per thread (jobs k and k + 256 of the block's 512), so every weight read from shared
// memory feeds both jobs' FMAs: the 64x64 layer's weights are read four at a time, and with one
// job per thread the shared-memory instruction queue, not the FMA pipe, bounds the kernel.  Each
// job's sums keep their order (each unit's row in order, y summed in unit order).
__global__ void __launch_bounds__(256, 1) predict_kernel(const float* __restrict__ params,
                                                      const float* __restrict__ feat, int n,
                                                      float* __restrict__ out) {
    __shared__ __align__(16) float w[kParams];
    for (int t = threadIdx.x; t < kParams; t += blockDim.x) w[t] = params[t];
    __syncthreads();
    const int ka = blockIdx.x * 2 * blockDim.x + threadIdx.x, kb = ka + blockDim.x;
    if (ka >= n) return;
    const bool has_b = kb < n;
    float xa[kF], xb[kF];
#pragma unroll
    for (int f = 0; f < kF; ++f) {
        xa[f] = feat[(size_t)ka * kF + f];
        xb[f] = has_b ? feat[(size_t)kb * kF + f] : 0.0f;
    }
    float ha[kH], hb[kH];
#pragma unroll
    for (int u = 0; u < kH; ++u) {
        float a = w[ob1 + u], b = a;
#pragma unroll
        for (int f = 0; f < kF; ++f) {
            const float c = w[oW1 + u * kF + f];
            a = fmaf(c, xa[f], a);
            b = fmaf(c, xb[f], b);
        }
        ha[u] = fmaxf(a, 0.0f);
        hb[u] = fmaxf(b, 0.0f);
    }
    // four hidden units at a time: four independent accumulation chains per job, rows of W2
    // four weights per broadcast load
    float ya = w[ob3], yb = ya;
    for (int u0 = 0; u0 < kH; u0 += 4) {
        float a[4], b[4];
        const float4* row[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            a[j] = b[j] = w[ob2 + u0 + j];
            row[j] = reinterpret_cast<const float4*>(w + oW2 + (u0 + j) * kH);
        }
#pragma unroll
        for (int q = 0; q < kH / 4; ++q) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float4 c = row[j][q];
                a[j] = fmaf(c.x, ha[4 * q], a[j]);
                b[j] = fmaf(c.x, hb[4 * q], b[j]);
                a[j] = fmaf(c.y, ha[4 * q + 1], a[j]);
                b[j] = fmaf(c.y, hb[4 * q + 1], b[j]);
                a[j] = fmaf(c.z, ha[4 * q + 2], a[j]);
                b[j] = fmaf(c.z, hb[4 * q + 2], b[j]);
                a[j] = fmaf(c.w, ha[4 * q + 3], a[j]);
                b[j] = fmaf(c.w, hb[4 * q + 3], b[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            ya = fmaf(w[oW3 + u0 + j], fmaxf(a[j], 0.0f), ya);
            yb = fmaf(w[oW3 + u0 + j], fmaxf(b[j], 0.0f), yb);
        }
    }
    out[ka] = ya;
    if (has_b) out[kb] = yb;
}

// ---- training: forward with saved activations, backward, Adam ----------------------------

// H1[b][u], H2[b][u] for a mini-batch, and dY[b] = 2 (Y - T) / B; loss partials per block.
__global__ void train_fwd_kernel(const float* __restrict__ p, const float* __restrict__ X,
                                 const float* __restrict__ T, const int* __restrict__ idx, int B,
                                 float* __restrict__ H1, float* __restrict__ H2,
                                 float* __restrict__ dY, float* __restrict__ loss_part) {
    __shared__ float w[kParams];
    __shared__ float red[256];
    for (int t = threadIdx.x; t < kParams; t += blockDim.x) w[t] = p[t];
    __syncthreads();
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    float sq = 0.0f;
    if (b < B) {
        const int s = idx ? idx[b] : b;
        float x[kF];
#pragma unroll
        for (int f = 0; f < kF; ++f) x[f] = X[(size_t)s * kF + f];
        float h1[kH];
#pragma unroll
        for (int u = 0; u < kH; ++u) {
            float a = w[ob1 + u];
#pragma unroll
            for (int f = 0; f < kF; ++f) a = fmaf(w[oW1 + u * kF + f], x[f], a);
            h1[u] = fmaxf(a, 0.0f);
            H1[(size_t)b * kH + u] = h1[u];
        }
        float y = w[ob3];
        for (int u = 0; u < kH; ++u) {
            float a = w[ob2 + u];
#pragma unroll
            for (int q = 0; q < kH; ++q) a = fmaf(w[oW2 + u * kH + q], h1[q], a);
            a = fmaxf(a, 0.0f);
            H2[(size_t)b * kH + u] = a;
            y = fmaf(w[oW3 + u], a, y);
        }
        const float e = y - T[s];
        dY[b] = 2.0f * e / (float)B;
        sq = e * e;
    }
    red[threadIdx.x] = sq;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0];
}

// dH2[b][u] = dY[b] * W3[u] * (H2 > 0);  dW3[u] = sum_b dY[b] H2[b][u]; db3 = sum_b dY[b]
__global__ void train_bwd3_kernel(const float* __restrict__ p, const float* __restrict__ H2,
                                  const float* __restrict__ dY, int B, float* __restrict__ dH2,
                                  float* __restrict__ g) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < B * kH) {
        const int b = t / kH, u = t % kH;
        dH2[t] = H2[t] > 0.0f ? dY[b] * p[oW3 + u] : 0.0f;
    }
    if (blockIdx.x == 0 && threadIdx.x <= kH) {
        float a = 0.0f;
        if (threadIdx.x < kH) {
            for (int b = 0; b < B; ++b) a = fmaf(dY[b], H2[(size_t)b * kH + threadIdx.x], a);
            g[oW3 + threadIdx.x] = a;
        } else {
            for (int b = 0; b < B; ++b) a += dY[b];
            g[ob3] = a;
        }
    }
}

// dW2[u][q] = sum_b dH2[b][u] H1[b][q];  db2[u] = sum_b dH2[b][u]
__global__ void train_gw2_kernel(const float* __restrict__ H1, const float* __restrict__ dH2,
                                 int B, float* __restrict__ g) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < kH * kH) {
        const int u = t / kH, q = t % kH;
        float a = 0.0f;
        for (int b = 0; b < B; ++b) a = fmaf(dH2[(size_t)b * kH + u], H1[(size_t)b * kH + q], a);
        g[oW2 + t] = a;
    } else if (t < kH * kH + kH) {
        const int u = t - kH * kH;
        float a = 0.0f;
        for (int b = 0; b < B; ++b) a += dH2[(size_t)b * kH + u];
        g[ob2 + u] = a;
    }
}

// dH1[b][q] = (sum_u dH2[b][u] W2[u][q]) * (H1 > 0)
__global__ void train_dh1_kernel(const float* __restrict__ p, const float* __restrict__ H1,
                                 const float* __restrict__ dH2, int B, float* __restrict__ dH1) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * kH) return;
    const int b = t / kH, q = t % kH;
    float a = 0.0f;
    for (int u = 0; u < kH; ++u) a = fmaf(dH2[(size_t)b * kH + u], p[oW2 + u * kH + q], a);
    dH1[t] = H1[t] > 0.0f ? a : 0.0f;
}

// dW1[u][f] = sum_b dH1[b][u] X[b][f];  db1[u] = sum_b dH1[b][u]
__global__ void train_gw1_kernel(const float* __restrict__ X, const int* __restrict__ idx,
                                 const float* __restrict__ dH1, int B, float* __restrict__ g) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < kH * kF) {
        const int u = t / kF, f = t % kF;
        float a = 0.0f;
        for (int b = 0; b < B; ++b) {
            const int s = idx ? idx[b] : b;
            a = fmaf(dH1[(size_t)b * kH + u], X[(size_t)s * kF + f], a);
        }
        g[oW1 + t] = a;
    } else if (t < kH * kF + kH) {
        const int u = t - kH * kF;
        float a = 0.0f;
        for (int b = 0; b < B; ++b) a += dH1[(size_t)b * kH + u];
        g[ob1 + u] = a;
    }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kParams) return;
    const float gg = g[t];
    const float mm = b1 * m[t] + (1.0f - b1) * gg;
    const float vv = b2 * v[t] + (1.0f - b2) * gg * gg;
    m[t] = mm;
    v[t] = vv;
    p[t] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

// Fisher-Yates shuffle of 0..n-1 with a splitmix64 stream, on one thread (n <= a few M).
__global__ void perm_kernel(int* __restrict__ idx, int n, unsigned long long seed) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int k = 0; k < n; ++k) idx[k] = k;
    unsigned long long s = seed;
    for (int k = n - 1; k > 0; --k) {
        unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const int j = (int)(z % (unsigned long long)(k + 1));
        const int tmp = idx[k]; idx[k] = idx[j]; idx[j] = tmp;
    }
}

// ---- host side ---------------------------------------------------------------------------

int model_features(const g3x_job_t* jobs, int n, const uint32_t* codes, const uint32_t* nmask,
                   int64_t n_bases, float* feat, cudaStream_t st, const int32_t* subset, const int32_t* subset_n) {
    if (n <= 0) return G3X_OK;
    features_kernel<<<(n + 255) / 256, 256, 0, st>>>(jobs, n, codes, nmask, n_bases, feat, subset, subset_n);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

int model_predict(const float* params, const float* feat, int n, float* out, cudaStream_t st) {
    if (n <= 0) return G3X_OK;
    predict_kernel<<<(n + 511) / 512, 256, 0, st>>>(params, feat, n, out);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

// ---- the learned schedule's keys: features, network and sort key in one kernel ----------

namespace {

// Two floats as a bf16 pair, rounded to nearest: x in the low half, y in the high half.
__device__ __forceinline__ uint32_t bf16x2(float x, float y) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(y), "f"(x));
    return r;
}

// D = A B + D on the tensor cores, m16n8k16, bf16 in, fp32 accumulate (PTX fragment layouts:
// a thread g = lane / 4, t = lane % 4 holds A rows g and g + 8 at columns 2t, 2t + 1 (registers 0,
// 1) and 2t + 8, 2t + 9 (registers 2, 3); B rows 2t, 2t + 1 and 2t + 8, 2t + 9 of column g; C rows
// g and g + 8 at columns 2t, 2t + 1).
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
                 "{%8,%9}, {%0,%1,%2,%3};"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

constexpr int kW2Stride = kH + 8;   // bf16 per row of W2 in shared memory (conflict-free B loads)

}  // namespace

// The learned schedule's sort keys (g3x_schedkey.cuh) with the network's prediction: one warp
// per 32 sort positions, each lane one job's features; the network runs on the tensor cores for
// each half-warp's 16 jobs (layer 1: 5 features padded to 16 columns by 64 units; layer 2: 64 by
// 64; both bf16 with fp32 sums, the biases and ReLUs in fp32), the 64 -> 1 layer as fp32 dot
// products reduced over the four lanes that hold a job's row.  In bf16 the prediction differs
// from g3x_mlp_predict's fp32 by a few hundredths of a log2 unit, a tenth of the row bin the key
// rounds it to.  Replaces three kernels of the learned schedule (features, network, keys) and
// their round trips through memory.  pred_out (optional) receives the corrections the keys use:
// the predictions, or 0 where near_diagonal keeps an early call in the length order.
__global__ void __launch_bounds__(128) learned_keys_kernel(const g3x_job_t* __restrict__ jobs, int n,
                                                           const uint32_t* __restrict__ codes,
                                                           const uint32_t* __restrict__ nmask, int64_t n_bases,
                                                           const float* __restrict__ params, ScoreParams sp,
                                                           TileTable tt, int32_t* __restrict__ bin,
                                                           int32_t* __restrict__ hist,
                                                           const int32_t* __restrict__ subset,
                                                           const int32_t* __restrict__ subset_n,
                                                           float* __restrict__ pred_out) {
    __shared__ uint32_t w1b[8][32];                  // layer-1 B fragments (register 0) per n-tile, lane
    __shared__ __align__(16) uint32_t w2s[kH * kW2Stride / 2];
    __shared__ float b1s[kH], b2s[kH], w3s[kH], b3s;
    for (int i = threadIdx.x; i < 8 * 32; i += blockDim.x) {
        const int nn = i >> 5, l = i & 31, u = 8 * nn + (l >> 2), f0 = 2 * (l & 3);
        const float x = f0 < kF ? params[oW1 + u * kF + f0] : 0.0f;
        const float y = f0 + 1 < kF ? params[oW1 + u * kF + f0 + 1] : 0.0f;
        w1b[nn][l] = bf16x2(x, y);
    }
    for (int i = threadIdx.x; i < kH * kH / 2; i += blockDim.x) {
        const int u = i / (kH / 2), c = 2 * (i % (kH / 2));
        w2s[(u * kW2Stride + c) / 2] = bf16x2(params[oW2 + u * kH + c], params[oW2 + u * kH + c + 1]);
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        b1s[i] = params[ob1 + i];
        b2s[i] = params[ob2 + i];
        w3s[i] = params[oW3 + i];
    }
    if (threadIdx.x == 0) b3s = params[ob3];
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int k0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31;   // the warp's first position
    const int cnt = subset_n ? min(n, *subset_n) : n;
    if (k0 >= cnt) return;                                         // the whole warp
    const int k = k0 + lane;
    const bool valid = k < cnt;
    const int job = valid ? (subset ? subset[k] : k) : 0;
    g3x_job_t jb = {};
    float f[kF] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    Head48 head;
    head.loaded = 0;
    if (valid) {
        jb = jobs[job];
        job_features(jb, codes, nmask, n_bases, f, &head);
    }
    const uint32_t p0 = bf16x2(f[0], f[1]), p1 = bf16x2(f[2], f[3]), p2 = bf16x2(f[4], 0.0f);
    float yv[2][2];                                   // [half-warp][row g, row g + 8]
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int ra = 16 * mt + g, rb = ra + 8;      // the lanes holding rows g and g + 8
        const uint32_t qa0 = __shfl_sync(0xFFFFFFFFu, p0, ra), qa1 = __shfl_sync(0xFFFFFFFFu, p1, ra),
                       qa2 = __shfl_sync(0xFFFFFFFFu, p2, ra);
        const uint32_t qb0 = __shfl_sync(0xFFFFFFFFu, p0, rb), qb1 = __shfl_sync(0xFFFFFFFFu, p1, rb),
                       qb2 = __shfl_sync(0xFFFFFFFFu, p2, rb);
        const uint32_t a1[4] = {t == 0 ? qa0 : t == 1 ? qa1 : t == 2 ? qa2 : 0u,
                                t == 0 ? qb0 : t == 1 ? qb1 : t == 2 ? qb2 : 0u, 0u, 0u};
        float h1[8][4];
#pragma unroll
        for (int nn = 0; nn < 8; ++nn) {
            const float bx = b1s[8 * nn + 2 * t], by = b1s[8 * nn + 2 * t + 1];
            h1[nn][0] = bx; h1[nn][1] = by; h1[nn][2] = bx; h1[nn][3] = by;
            mma_bf16(h1[nn], a1, w1b[nn][lane], 0u);
#pragma unroll
            for (int e = 0; e < 4; ++e) h1[nn][e] = fmaxf(h1[nn][e], 0.0f);
        }
        float h2[8][4];
#pragma unroll
        for (int nn = 0; nn < 8; ++nn) {
            const float bx = b2s[8 * nn + 2 * t], by = b2s[8 * nn + 2 * t + 1];
            h2[nn][0] = bx; h2[nn][1] = by; h2[nn][2] = bx; h2[nn][3] = by;
        }
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            // layer 1's C fragments of n-tiles 2kk, 2kk + 1 are layer 2's A fragment of k-step kk
            const uint32_t a2[4] = {bf16x2(h1[2 * kk][0], h1[2 * kk][1]), bf16x2(h1[2 * kk][2], h1[2 * kk][3]),
                                    bf16x2(h1[2 * kk + 1][0], h1[2 * kk + 1][1]),
                                    bf16x2(h1[2 * kk + 1][2], h1[2 * kk + 1][3])};
#pragma unroll
            for (int nn = 0; nn < 8; ++nn) {
                const uint32_t* row = w2s + (8 * nn + g) * (kW2Stride / 2);
                mma_bf16(h2[nn], a2, row[8 * kk + t], row[8 * kk + t + 4]);
            }
        }
        float ylo = 0.0f, yhi = 0.0f;
#pragma unroll
        for (int nn = 0; nn < 8; ++nn) {
            const float wx = w3s[8 * nn + 2 * t], wy = w3s[8 * nn + 2 * t + 1];
            ylo = fmaf(wx, fmaxf(h2[nn][0], 0.0f), ylo);
            ylo = fmaf(wy, fmaxf(h2[nn][1], 0.0f), ylo);
            yhi = fmaf(wx, fmaxf(h2[nn][2], 0.0f), yhi);
            yhi = fmaf(wy, fmaxf(h2[nn][3], 0.0f), yhi);
        }
        ylo += __shfl_xor_sync(0xFFFFFFFFu, ylo, 1);
        ylo += __shfl_xor_sync(0xFFFFFFFFu, ylo, 2);
        yhi += __shfl_xor_sync(0xFFFFFFFFu, yhi, 1);
        yhi += __shfl_xor_sync(0xFFFFFFFFu, yhi, 2);
        yv[mt][0] = ylo + b3s;
        yv[mt][1] = yhi + b3s;
    }
    // the lane's own job: row r = lane % 16 of half-warp lane / 16, held by lane 4 (r % 8)
    const int r = lane & 15, src = (r & 7) << 2;
    const float v00 = __shfl_sync(0xFFFFFFFFu, yv[0][0], src), v01 = __shfl_sync(0xFFFFFFFFu, yv[0][1], src);
    const float v10 = __shfl_sync(0xFFFFFFFFu, yv[1][0], src), v11 = __shfl_sync(0xFFFFFFFFu, yv[1][1], src);
    const float pr = lane < 16 ? (r < 8 ? v00 : v01) : (r < 8 ? v10 : v11);
    // a job the network calls early-ending stays in the length order when a diagonal next to the
    // seed's continues the alignment (near_diagonal)
    const float corr = valid && pr + kLearnedSlack < 0.0f && near_diagonal(jb, codes, nmask, n_bases, head) ? 0.0f : pr;
    if (valid) {
        if (pred_out) pred_out[job] = corr;
        const int bn = sched_key(jb, sp, tt, true, corr);
        bin[k] = bn;
        sched_count(hist, bn);
    }
}

int launch_learned_keys(const float* params, const g3x_job_t* jobs, int n, const uint32_t* codes,
                        const uint32_t* nmask, int64_t n_bases, const ScoreParams& sp, const TileTable& tt,
                        int32_t* bin, int32_t* hist, cudaStream_t st, const int32_t* subset,
                        const int32_t* subset_n, float* pred_out) {
    if (n <= 0) return G3X_OK;
    learned_keys_kernel<<<(n + 127) / 128, 128, 0, st>>>(jobs, n, codes, nmask, n_bases, params, sp, tt, bin, hist,
                                                         subset, subset_n, pred_out);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

// One mini-batch gradient into g (and the batch's squared-error sum in *loss_sum_dev).
static int batch_grad(ModelState& M, const float* X, const float* T, const int* idx, int B,
                      cudaStream_t st) {
    const int nb = (B + 255) / 256;
    train_fwd_kernel<<<nb, 256, 0, st>>>(M.params, X, T, idx, B, M.h1, M.h2, M.dy, M.loss_part);
    train_bwd3_kernel<<<(B * kH + 255) / 256, 256, 0, st>>>(M.params, M.h2, M.dy, B, M.dh2, M.grad);
    train_gw2_kernel<<<(kH * kH + kH + 255) / 256, 256, 0, st>>>(M.h1, M.dh2, B, M.grad);
    train_dh1_kernel<<<(B * kH + 255) / 256, 256, 0, st>>>(M.params, M.h1, M.dh2, B, M.dh1);
    train_gw1_kernel<<<(kH * kF + kH + 255) / 256, 256, 0, st>>>(X, idx, M.dh1, B, M.grad);
    return cudaPeekAtLastError() == cudaSuccess ? G3X_OK : G3X_ERR_CUDA;
}

int model_alloc(ModelState& M, int batch) {
    if (M.params && batch <= M.batch_cap) return G3X_OK;
    if (!M.params) {
        if (cudaMalloc(&M.params, kParams * sizeof(float)) || cudaMalloc(&M.grad, kParams * sizeof(float)) ||
            cudaMalloc(&M.m, kParams * sizeof(float)) || cudaMalloc(&M.v, kParams * sizeof(float)))
            return G3X_ERR_NOMEM;
        cudaMemset(M.params, 0, kParams * sizeof(float));
    }
    cudaFree(M.h1); cudaFree(M.h2); cudaFree(M.dh1); cudaFree(M.dh2); cudaFree(M.dy);
    cudaFree(M.loss_part);
    const size_t b = (size_t)batch;
    if (cudaMalloc(&M.h1, b * kH * sizeof(float)) || cudaMalloc(&M.h2, b * kH * sizeof(float)) ||
        cudaMalloc(&M.dh1, b * kH * sizeof(float)) || cudaMalloc(&M.dh2, b * kH * sizeof(float)) ||
        cudaMalloc(&M.dy, b * sizeof(float)) ||
        cudaMalloc(&M.loss_part, ((b + 255) / 256) * sizeof(float)))
        return G3X_ERR_NOMEM;
    M.batch_cap = batch;
    return G3X_OK;
}

void model_free(ModelState& M) {
    cudaFree(M.params); cudaFree(M.grad); cudaFree(M.m); cudaFree(M.v);
    cudaFree(M.h1); cudaFree(M.h2); cudaFree(M.dh1); cudaFree(M.dh2); cudaFree(M.dy);
    cudaFree(M.loss_part); cudaFree(M.perm);
    M = ModelState();
}

int model_gradient(ModelState& M, const float* X, const float* T, int B, float* h_grad,
                   float* h_loss, cudaStream_t st) {
    int rc = model_alloc(M, B);
    if (rc) return rc;
    if ((rc = batch_grad(M, X, T, nullptr, B, st))) return rc;
    const int nb = (B + 255) / 256;
    float* lp = new float[nb];
    if (cudaMemcpyAsync(h_grad, M.grad, kParams * sizeof(float), cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(lp, M.loss_part, nb * sizeof(float), cudaMemcpyDeviceToHost, st) ||
        cudaStreamSynchronize(st)) {
        delete[] lp;
        return G3X_ERR_CUDA;
    }
    double s = 0;
    for (int k = 0; k < nb; ++k) s += lp[k];
    delete[] lp;
    if (h_loss) *h_loss = (float)(s / B);
    return G3X_OK;
}

int model_train(ModelState& M, const float* X, const float* T, int n, int epochs, int batch,
                float lr, uint64_t seed, float* h_epoch_loss, cudaStream_t st) {
    if (batch <= 0 || n < batch) return G3X_ERR_INVALID;
    int rc = model_alloc(M, batch);
    if (rc) return rc;
    if (n > M.perm_cap) {
        cudaFree(M.perm);
        if (cudaMalloc(&M.perm, (size_t)n * sizeof(int))) return G3X_ERR_NOMEM;
        M.perm_cap = n;
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const int steps = n / batch;
    const int nb = (batch + 255) / 256;
    float* lp = new float[nb];
    for (int ep = 0; ep < epochs; ++ep) {
        perm_kernel<<<1, 1, 0, st>>>(M.perm, n, seed * 1000003ull + (unsigned long long)ep);
        double loss = 0;
        for (int s = 0; s < steps; ++s) {
            if ((rc = batch_grad(M, X, T, M.perm + (size_t)s * batch, batch, st))) break;
            ++M.t;
            const float c1 = 1.0f - powf(b1, (float)M.t), c2 = 1.0f - powf(b2, (float)M.t);
            adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(M.params, M.grad, M.m, M.v, lr, b1, b2, eps, c1, c2);
            if (h_epoch_loss && s == steps - 1) {
                if (cudaMemcpyAsync(lp, M.loss_part, nb * sizeof(float), cudaMemcpyDeviceToHost, st) ||
                    cudaStreamSynchronize(st)) { rc = G3X_ERR_CUDA; break; }
                for (int k = 0; k < nb; ++k) loss += lp[k];
            }
        }
        if (rc) break;
        if (h_epoch_loss) h_epoch_loss[ep] = (float)(loss / batch);
    }
    delete[] lp;
    if (rc == G3X_OK && cudaPeekAtLastError() != cudaSuccess) rc = G3X_ERR_CUDA;
    return rc;
}

// He-style initialisation from a splitmix64 stream (host), Adam state zeroed.
int model_init(ModelState& M, uint64_t seed) {
    int rc = model_alloc(M, 256);
    if (rc) return rc;
    float* h = new float[kParams];
    uint64_t s = seed;
    auto uni = [&]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (float)((double)(z >> 11) * (1.0 / 9007199254740992.0)) * 2.0f - 1.0f;
    };
    for (int k = 0; k < kParams; ++k) h[k] = 0.0f;
    for (int k = 0; k < kH * kF; ++k) h[oW1 + k] = uni() * sqrtf(6.0f / kF);
    for (int k = 0; k < kH * kH; ++k) h[oW2 + k] = uni() * sqrtf(6.0f / kH);
    for (int k = 0; k < kH; ++k) h[oW3 + k] = uni() * sqrtf(3.0f / kH);
    rc = cudaMemcpy(M.params, h, kParams * sizeof(float), cudaMemcpyHostToDevice) ? G3X_ERR_CUDA : G3X_OK;
    delete[] h;
    cudaMemset(M.m, 0, kParams * sizeof(float));
    cudaMemset(M.v, 0, kParams * sizeof(float));
    M.t = 0;
    M.trained = rc == G3X_OK ? 0 : M.trained;
    return rc;
}

}  // namespace g3x
