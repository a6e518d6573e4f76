// Learned block proposal: spectrogram, BF16 tensor-core inference (mma.sync
// m16n8k16, FP32 accumulation) and FP32 training kernels (proposal.hpp).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "common.cuh"
#include "proposal.hpp"

namespace empi {

// ------------------------------------------------------------ spectrogram
//
// 128 frames of 2 ceil(N / 128) samples (Hann window, centres (i + 1/2) N / 128),
// 64 bins at (k + 1/2) / 128 cycles per sample (0 .. fs / 2), power summed over
// the instance's channels, log, then per instance zero mean and unit variance
// (so the input does not depend on the signal's amplitude).
// out + inst * inst_stride (+ the instance's iteration * 64 * 128 with per_it:
// one spectrogram per MP iteration, the training pairs' inputs)
__device__ __forceinline__ float* spec_at(float* out, const InstState& st, int inst, long long inst_stride,
                                          int per_it) {
    return out + (long long)inst * inst_stride + (per_it ? (long long)st.it * kSpecSize : 0);
}

// One CTA per (frame, instance), a thread per bin.  The frame's Hann-windowed
// samples are staged in shared memory kSpecStage at a time (the window once
// per sample, not once per bin and sample); each bin's twiddle e^{-2 pi i nu m}
// is rotated from sample to sample and set exactly at every stage's start,
// so the rotation's rounding stays at the 1e-5 level of a heuristic input.
constexpr int kSpecStage = 256;

__global__ void k_spectrogram(BatchDev b, float* out, long long inst_stride, int per_it) {
    __shared__ float sv[kSpecStage];
    const int inst = blockIdx.y, frame = blockIdx.x, k = threadIdx.x;
    const InstState& st = b.state[inst];
    if (st.status != ST_RUNNING || (per_it && st.it >= b.iter_max)) return;
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    const int N = dp.N;
    const int Wf = max(4, 2 * ((N + kSpecT - 1) / kSpecT));
    const int c0 = (int)(((long long)(2 * frame + 1) * N) / (2 * kSpecT));
    const int n0 = c0 - Wf / 2;
    const float nu = (k + 0.5f) / (2.0f * kSpecF);  // cycles per sample
    float stp_s, stp_c;
    sincospif(-2.0f * nu, &stp_s, &stp_c);
    const float2 step = make_float2(stp_c, stp_s);
    float pw = 0.0f;
    for (int c = 0; c < ip.C; ++c) {
        const float* x = b.residual32 + ip.res_off + (long long)c * N;
        float ar = 0.0f, ai = 0.0f;
        for (int m0 = 0; m0 < Wf; m0 += kSpecStage) {
            const int len = min(kSpecStage, Wf - m0);
            __syncthreads();  // the previous stage's samples are consumed
            for (int i = k; i < len; i += blockDim.x) {
                const int m = m0 + i, n = n0 + m;
                const float w = 0.5f - 0.5f * cospif(2.0f * (m + 0.5f) / (float)Wf);
                sv[i] = (n >= 0 && n < N) ? x[n] * w : 0.0f;
            }
            __syncthreads();
            float ts, tc;
            sincospif(-2.0f * nu * (float)m0, &ts, &tc);
            float2 t = make_float2(tc, ts);
            for (int i = 0; i < len; ++i) {
                const float v = sv[i];
                ar += v * t.x;
                ai += v * t.y;
                t = make_float2(t.x * step.x - t.y * step.y, t.x * step.y + t.y * step.x);
            }
        }
        pw += ar * ar + ai * ai;
    }
    spec_at(out, st, inst, inst_stride, per_it)[k * kSpecT + frame] = logf(pw + 1e-30f);
}

// per instance: zero mean, unit variance over the 64 x 128 values
__global__ void k_spec_normalise(float* spec, const InstState* state, int iter_max, long long inst_stride,
                                 int per_it) {
    __shared__ float red[2][32];
    const int inst = blockIdx.x;
    const InstState& st = state[inst];
    if (st.status != ST_RUNNING || (per_it && st.it >= iter_max)) return;
    float* x = spec_at(spec, st, inst, inst_stride, per_it);
    float s = 0.0f, q = 0.0f;
    for (int i = threadIdx.x; i < kSpecSize; i += blockDim.x) {
        s += x[i];
        q += x[i] * x[i];
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, off);
        q += __shfl_down_sync(0xffffffffu, q, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = s;
        red[1][threadIdx.x >> 5] = q;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float ts = 0.0f, tq = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            ts += red[0][w];
            tq += red[1][w];
        }
        red[0][0] = ts / kSpecSize;
        red[1][0] = tq / kSpecSize;
    }
    __syncthreads();
    const float mean = red[0][0];
    const float var = fmaxf(red[1][0] - mean * mean, 0.0f);
    const float inv = var > 0.0f ? rsqrtf(var) : 1.0f;
    for (int i = threadIdx.x; i < kSpecSize; i += blockDim.x) x[i] = (x[i] - mean) * inv;
}

// ------------------------------------------------------------ layers as GEMMs
//
// Every layer is out[n][m] = act(sum_k A[m][k] W[n][k] + bias[n]) over the
// layer's output positions m, outputs n and inputs k: a 3x3 convolution reads
// A[m][k] = in[ci][oy S - 1 + ky][ox S - 1 + kx] (zero outside) with
// k = (ci, ky, kx), m = (oy, ox); the last layer reads A[m][k] = x3[k][m]
// (k = (channel, frequency), m = time column).
template <int CIN_, int HIN_, int WIN_, int STRIDE_, int COUT_, bool DENSE_, bool RELU_>
struct Layer {
    static constexpr int CIN = CIN_, HIN = HIN_, WIN = WIN_, STRIDE = STRIDE_, COUT = COUT_;
    static constexpr bool DENSE = DENSE_, RELU = RELU_;
    static constexpr int HOUT = DENSE ? 1 : HIN / STRIDE, WOUT = DENSE ? WIN : WIN / STRIDE;
    static constexpr int M = HOUT * WOUT;
    static constexpr int K = DENSE ? CIN * HIN : CIN * 9;
    static constexpr int KP = (K + 15) / 16 * 16;  // padded to the MMA's k = 16
    static constexpr int IN_SIZE = CIN * HIN * WIN, OUT_SIZE = COUT * M;
    __device__ __forceinline__ static float a(const float* in, int m, int k) {
        if (k >= K) return 0.0f;
        if (DENSE) return in[k * WIN + m];
        const int ci = k / 9, r = k - ci * 9, ky = r / 3, kx = r - ky * 3;
        const int oy = m / WOUT, ox = m - oy * WOUT;
        const int iy = oy * STRIDE - 1 + ky, ix = ox * STRIDE - 1 + kx;
        return (iy >= 0 && iy < HIN && ix >= 0 && ix < WIN) ? in[(ci * HIN + iy) * WIN + ix] : 0.0f;
    }
};

using L1 = Layer<1, kSpecF, kSpecT, 1, kC1, false, true>;
using L2 = Layer<kC1, kH1, kW1n, 2, kC2, false, true>;
using L3 = Layer<kC2, kH2, kW2n, 2, kC3, false, true>;
using L4 = Layer<kC3, kH3, kW3n, 1, kBands, true, false>;
static_assert(L1::OUT_SIZE == kAct1 && L2::OUT_SIZE == kAct2 && L3::OUT_SIZE == kAct3 && L4::OUT_SIZE == kScores,
              "layer shapes");
static_assert(L1::COUT * L1::K + L1::COUT == kOffW2 && kOffW3 - kOffW2 == L2::COUT * L2::K + L2::COUT &&
                  kOffW4 - kOffW3 == L3::COUT * L3::K + L3::COUT && kNetParams - kOffW4 == L4::COUT * L4::K + L4::COUT,
              "parameter layout");

// ------------------------------------------------------------ BF16 tensor-core inference
//
// One warp computes a 16-position x COUT tile with mma.sync m16n8k16 (BF16
// inputs, FP32 accumulation): per k step it builds its A fragment (rows g and
// g + 8 of the tile, columns 2 t, 2 t + 1 and 2 t + 8, 2 t + 9; g = lane / 4,
// t = lane % 4) from the layer's input, and reads B (W[n][k], n = g) from
// the layer's BF16 weights staged in shared memory as [COUT][KP].
__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // lo in the low half
    return *reinterpret_cast<const unsigned*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template <class LY>
__global__ void __launch_bounds__(128) k_layer_bf16(const float* in, long long in_stride, float* out,
                                                     long long out_stride, const __nv_bfloat16* w, const float* bias,
                                                     const InstState* state) {
    static_assert(LY::M % 16 == 0 && LY::COUT % 8 == 0, "tile shapes");
    __shared__ __align__(16) __nv_bfloat16 sw[LY::COUT * LY::KP];
    const int inst = blockIdx.y;
    if (state && state[inst].status != ST_RUNNING) return;  // the whole CTA
    for (int i = threadIdx.x; i < LY::COUT * LY::KP; i += blockDim.x) sw[i] = w[i];
    __syncthreads();
    const float* x = in + (long long)inst * in_stride;
    float* y = out + (long long)inst * out_stride;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
    constexpr int NT = LY::COUT / 8;
    for (int mt = (blockIdx.x * 4 + warp) * 16; mt < LY::M; mt += gridDim.x * 4 * 16) {
        float acc[NT][4];
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
        const int r0 = mt + g, r1 = mt + g + 8;
        for (int k0 = 0; k0 < LY::KP; k0 += 16) {
            const int ka = k0 + tg * 2, kb = ka + 8;
            const unsigned a0 = pack_bf16(LY::a(x, r0, ka), LY::a(x, r0, ka + 1));
            const unsigned a1 = pack_bf16(LY::a(x, r1, ka), LY::a(x, r1, ka + 1));
            const unsigned a2 = pack_bf16(LY::a(x, r0, kb), LY::a(x, r0, kb + 1));
            const unsigned a3 = pack_bf16(LY::a(x, r1, kb), LY::a(x, r1, kb + 1));
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const __nv_bfloat16* wn = sw + (nt * 8 + g) * LY::KP;
                const unsigned b0 = *reinterpret_cast<const unsigned*>(wn + ka);
                const unsigned b1 = *reinterpret_cast<const unsigned*>(wn + kb);
                mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
            }
        }
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int n0 = nt * 8 + tg * 2;
            float v[4] = {acc[nt][0] + bias[n0], acc[nt][1] + bias[n0 + 1], acc[nt][2] + bias[n0],
                          acc[nt][3] + bias[n0 + 1]};
            if (LY::RELU)
                for (int i = 0; i < 4; ++i) v[i] = fmaxf(v[i], 0.0f);
            y[n0 * LY::M + r0] = v[0];
            y[(n0 + 1) * LY::M + r0] = v[1];
            y[n0 * LY::M + r1] = v[2];
            y[(n0 + 1) * LY::M + r1] = v[3];
        }
    }
}

// ------------------------------------------------------------ FP32 forward and backward (training)
//
// Batched over n samples (sample s reads in + order[s] * in_stride when an
// order is given, else in + s * in_stride): plain FP32 arithmetic, one thread
// per output value.
template <class LY>
__global__ void k_layer_f32(const float* in, long long in_stride, const int* order, float* out, const float* w,
                            const float* bias, int n) {
    const long long total = (long long)n * LY::COUT * LY::M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / (LY::COUT * LY::M));
        const int r = (int)(i - (long long)s * LY::COUT * LY::M);
        const int nn = r / LY::M, m = r - nn * LY::M;
        const float* x = in + (long long)(order ? order[s] : s) * in_stride;
        float acc = bias[nn];
        const float* wn = w + nn * LY::K;
        for (int k = 0; k < LY::K; ++k) acc += LY::a(x, m, k) * wn[k];
        out[i] = LY::RELU ? fmaxf(acc, 0.0f) : acc;
    }
}

// dOut -> dPre through the ReLU (out > 0), in place
__global__ void k_relu_back(float* d, const float* out, long long total) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
        if (!(out[i] > 0.0f)) d[i] = 0.0f;
}

// dW[n][k] += sum_m dPre_s[n][m] A_s[m][k] (one sample per blockIdx.y), dB[n] likewise
template <class LY>
__global__ void k_layer_dw(const float* in, long long in_stride, const int* order, const float* dpre, float* dw,
                           float* db) {
    const int s = blockIdx.y;
    const float* x = in + (long long)(order ? order[s] : s) * in_stride;
    const float* d = dpre + (long long)s * LY::COUT * LY::M;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < LY::COUT * (LY::K + 1); i += gridDim.x * blockDim.x) {
        const int nn = i / (LY::K + 1), k = i - nn * (LY::K + 1);
        const float* dn = d + nn * LY::M;
        float acc = 0.0f;
        if (k == LY::K) {
            for (int m = 0; m < LY::M; ++m) acc += dn[m];
            atomicAdd(db + nn, acc);
        } else {
            for (int m = 0; m < LY::M; ++m) acc += dn[m] * LY::a(x, m, k);
            atomicAdd(dw + nn * LY::K + k, acc);
        }
    }
}

// dIn = the transpose of the layer applied to dPre (one thread per input value)
template <class LY>
__global__ void k_layer_dx(const float* dpre, const float* w, float* din, int n) {
    const long long total = (long long)n * LY::IN_SIZE;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / LY::IN_SIZE);
        const int r = (int)(i - (long long)s * LY::IN_SIZE);
        const float* d = dpre + (long long)s * LY::COUT * LY::M;
        float acc = 0.0f;
        if (LY::DENSE) {
            const int k = r / LY::WIN, m = r - k * LY::WIN;
            for (int nn = 0; nn < LY::COUT; ++nn) acc += d[nn * LY::M + m] * w[nn * LY::K + k];
        } else {
            const int ci = r / (LY::HIN * LY::WIN), rr = r - ci * LY::HIN * LY::WIN;
            const int iy = rr / LY::WIN, ix = rr - iy * LY::WIN;
            for (int ky = 0; ky < 3; ++ky) {
                const int ny = iy + 1 - ky;
                if (ny < 0 || ny % LY::STRIDE) continue;
                const int oy = ny / LY::STRIDE;
                if (oy >= LY::HOUT) continue;
                for (int kx = 0; kx < 3; ++kx) {
                    const int nx = ix + 1 - kx;
                    if (nx < 0 || nx % LY::STRIDE) continue;
                    const int ox = nx / LY::STRIDE;
                    if (ox >= LY::WOUT) continue;
                    const int m = oy * LY::WOUT + ox, k = ci * 9 + ky * 3 + kx;
                    for (int nn = 0; nn < LY::COUT; ++nn) acc += d[nn * LY::M + m] * w[nn * LY::K + k];
                }
            }
        }
        din[i] = acc;
    }
}

// softmax cross-entropy over the 512 block scores of each sample: the loss
// (summed into loss[0]) and dScores = (softmax - onehot(label)) / n
__global__ void k_softmax_ce(const float* scores, const int* labels, const int* order, int n, float* dscores,
                             float* loss) {
    __shared__ float red[32];
    const int s = blockIdx.x;
    const float* z = scores + (long long)s * kScores;
    float mx = -3.0e38f;
    for (int i = threadIdx.x; i < kScores; i += blockDim.x) mx = fmaxf(mx, z[i]);
#pragma unroll
    for (int off = 16; off; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) t = fmaxf(t, red[w]);
        red[0] = t;
    }
    __syncthreads();
    mx = red[0];
    __syncthreads();
    float se = 0.0f;
    for (int i = threadIdx.x; i < kScores; i += blockDim.x) se += expf(z[i] - mx);
#pragma unroll
    for (int off = 16; off; off >>= 1) se += __shfl_xor_sync(0xffffffffu, se, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = se;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        red[0] = t;
    }
    __syncthreads();
    const float lse = mx + logf(red[0]);
    const int label = labels[order ? order[s] : s];
    for (int i = threadIdx.x; i < kScores; i += blockDim.x)
        dscores[(long long)s * kScores + i] = (expf(z[i] - lse) - (i == label ? 1.0f : 0.0f)) / (float)n;
    if (threadIdx.x == 0) atomicAdd(loss, (lse - z[label]) / (float)n);
}

// SGD with momentum: v = mu v + g, w -= lr v
__global__ void k_sgd(float* w, float* v, const float* g, int count, float lr, float mu) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        v[i] = mu * v[i] + g[i];
        w[i] -= lr * v[i];
    }
}

// ------------------------------------------------------------ host side

namespace {

constexpr size_t kBf1 = 0, kBf2 = kBf1 + (size_t)L1::COUT * L1::KP, kBf3 = kBf2 + (size_t)L2::COUT * L2::KP,
                 kBf4 = kBf3 + (size_t)L3::COUT * L3::KP, kBfAll = kBf4 + (size_t)L4::COUT * L4::KP;
constexpr int kBias1 = 0, kBias2 = kBias1 + L1::COUT, kBias3 = kBias2 + L2::COUT, kBias4 = kBias3 + L3::COUT,
              kBiasAll = kBias4 + L4::COUT;
constexpr long long kActAll = (long long)kAct1 + kAct2 + kAct3;

bool cuda_ok(cudaError_t e, std::string* err, const char* what) {
    if (e == cudaSuccess) return true;
    if (err) *err = std::string("cuda: ") + cudaGetErrorString(e) + " (" + what + ")";
    return false;
}

template <class LY>
void layer_to_bf16(const float* weights, int woff, std::vector<__nv_bfloat16>& out) {
    for (int n = 0; n < LY::COUT; ++n)
        for (int k = 0; k < LY::KP; ++k)
            out.push_back(__float2bfloat16(k < LY::K ? weights[woff + n * LY::K + k] : 0.0f));
}

// BF16 GEMM layouts [COUT][KP] of the four layers, and their FP32 biases
void device_layouts(const float* w, std::vector<__nv_bfloat16>& bf, std::vector<float>& bias) {
    bf.clear();
    bf.reserve(kBfAll);
    layer_to_bf16<L1>(w, kOffW1, bf);
    layer_to_bf16<L2>(w, kOffW2, bf);
    layer_to_bf16<L3>(w, kOffW3, bf);
    layer_to_bf16<L4>(w, kOffW4, bf);
    bias.assign(w + kOffB1, w + kOffB1 + L1::COUT);
    bias.insert(bias.end(), w + kOffB2, w + kOffB2 + L2::COUT);
    bias.insert(bias.end(), w + kOffB3, w + kOffB3 + L3::COUT);
    bias.insert(bias.end(), w + kOffB4, w + kOffB4 + L4::COUT);
}

int grid_m(int m) { return std::max(1, std::min(128, (m + 63) / 64)); }

// BF16 inference of `ninst` spectrograms (spec + i * spec_stride) into
// scores [inst][512]; instances whose state is not running are skipped
void forward_bf16(const float* spec, long long spec_stride, float* act, const __nv_bfloat16* w, const float* bias,
                  float* scores, int ninst, const InstState* state, cudaStream_t s) {
    k_layer_bf16<L1><<<dim3(grid_m(L1::M), ninst), 128, 0, s>>>(spec, spec_stride, act, kActAll, w + kBf1,
                                                                  bias + kBias1, state);
    k_layer_bf16<L2><<<dim3(grid_m(L2::M), ninst), 128, 0, s>>>(act, kActAll, act + kAct1, kActAll, w + kBf2,
                                                                  bias + kBias2, state);
    k_layer_bf16<L3><<<dim3(grid_m(L3::M), ninst), 128, 0, s>>>(act + kAct1, kActAll, act + kAct1 + kAct2, kActAll,
                                                                  w + kBf3, bias + kBias3, state);
    k_layer_bf16<L4><<<dim3(grid_m(L4::M), ninst), 128, 0, s>>>(act + kAct1 + kAct2, kActAll, scores, kScores,
                                                                  w + kBf4, bias + kBias4, state);
}

int grid_for(long long n) { return (int)std::max<long long>(1, std::min<long long>(148 * 16, (n + 255) / 256)); }

// FP32 forward, backward and SGD over minibatches of host-provided pairs
struct Trainer {
    int cap = 0;  // samples per step
    float *spec = nullptr, *w = nullptr, *v = nullptr, *g = nullptr, *a1 = nullptr, *a2 = nullptr, *a3 = nullptr,
          *sc = nullptr, *d1 = nullptr, *d2 = nullptr, *d3 = nullptr, *dsc = nullptr, *loss = nullptr;
    int *labels = nullptr, *order = nullptr;
    std::string* err;
    explicit Trainer(std::string* e) : err(e) {}
    ~Trainer() {
        for (float* p : {spec, w, v, g, a1, a2, a3, sc, d1, d2, d3, dsc, loss})
            if (p) cudaFree(p);
        if (labels) cudaFree(labels);
        if (order) cudaFree(order);
    }
    bool init(const float* hspec, const int* hlabels, int n, int step_cap, const float* weights) {
        cap = step_cap;
        return cuda_ok(cudaMalloc(&spec, sizeof(float) * (size_t)n * kSpecSize), err, "spec") &&
               cuda_ok(cudaMemcpy(spec, hspec, sizeof(float) * (size_t)n * kSpecSize, cudaMemcpyHostToDevice), err,
                       "spec") &&
               cuda_ok(cudaMalloc(&labels, sizeof(int) * (size_t)std::max(n, 1)), err, "labels") &&
               (!hlabels || cuda_ok(cudaMemcpy(labels, hlabels, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice), err,
                                    "labels")) &&
               cuda_ok(cudaMalloc(&w, sizeof(float) * kNetParams), err, "w") &&
               cuda_ok(cudaMemcpy(w, weights, sizeof(float) * kNetParams, cudaMemcpyHostToDevice), err, "w") &&
               cuda_ok(cudaMalloc(&v, sizeof(float) * kNetParams), err, "v") &&
               cuda_ok(cudaMemset(v, 0, sizeof(float) * kNetParams), err, "v") &&
               cuda_ok(cudaMalloc(&g, sizeof(float) * kNetParams), err, "g") &&
               cuda_ok(cudaMalloc(&a1, sizeof(float) * (size_t)cap * kAct1), err, "a1") &&
               cuda_ok(cudaMalloc(&a2, sizeof(float) * (size_t)cap * kAct2), err, "a2") &&
               cuda_ok(cudaMalloc(&a3, sizeof(float) * (size_t)cap * kAct3), err, "a3") &&
               cuda_ok(cudaMalloc(&sc, sizeof(float) * (size_t)cap * kScores), err, "sc") &&
               cuda_ok(cudaMalloc(&d1, sizeof(float) * (size_t)cap * kAct1), err, "d1") &&
               cuda_ok(cudaMalloc(&d2, sizeof(float) * (size_t)cap * kAct2), err, "d2") &&
               cuda_ok(cudaMalloc(&d3, sizeof(float) * (size_t)cap * kAct3), err, "d3") &&
               cuda_ok(cudaMalloc(&dsc, sizeof(float) * (size_t)cap * kScores), err, "dsc") &&
               cuda_ok(cudaMalloc(&loss, sizeof(float)), err, "loss") &&
               cuda_ok(cudaMalloc(&order, sizeof(int) * (size_t)cap), err, "order");
    }
    void forward(int nb) {
        k_layer_f32<L1><<<grid_for((long long)nb * kAct1), 256>>>(spec, kSpecSize, order, a1, w + kOffW1,
                                                                  w + kOffB1, nb);
        k_layer_f32<L2><<<grid_for((long long)nb * kAct2), 256>>>(a1, kAct1, nullptr, a2, w + kOffW2, w + kOffB2, nb);
        k_layer_f32<L3><<<grid_for((long long)nb * kAct3), 256>>>(a2, kAct2, nullptr, a3, w + kOffW3, w + kOffB3, nb);
        k_layer_f32<L4><<<grid_for((long long)nb * kScores), 256>>>(a3, kAct3, nullptr, sc, w + kOffW4, w + kOffB4,
                                                                    nb);
    }
    // gradient of the mean loss over the nb samples in `order` into g, loss into loss[0]
    void gradients(int nb) {
        cudaMemset(g, 0, sizeof(float) * kNetParams);
        cudaMemset(loss, 0, sizeof(float));
        forward(nb);
        k_softmax_ce<<<nb, 128>>>(sc, labels, order, nb, dsc, loss);
        const dim3 gw(64, nb);
        k_layer_dw<L4><<<gw, 256>>>(a3, kAct3, nullptr, dsc, g + kOffW4, g + kOffB4);
        k_layer_dx<L4><<<grid_for((long long)nb * kAct3), 256>>>(dsc, w + kOffW4, d3, nb);
        k_relu_back<<<grid_for((long long)nb * kAct3), 256>>>(d3, a3, (long long)nb * kAct3);
        k_layer_dw<L3><<<gw, 256>>>(a2, kAct2, nullptr, d3, g + kOffW3, g + kOffB3);
        k_layer_dx<L3><<<grid_for((long long)nb * kAct2), 256>>>(d3, w + kOffW3, d2, nb);
        k_relu_back<<<grid_for((long long)nb * kAct2), 256>>>(d2, a2, (long long)nb * kAct2);
        k_layer_dw<L2><<<gw, 256>>>(a1, kAct1, nullptr, d2, g + kOffW2, g + kOffB2);
        k_layer_dx<L2><<<grid_for((long long)nb * kAct1), 256>>>(d2, w + kOffW2, d1, nb);
        k_relu_back<<<grid_for((long long)nb * kAct1), 256>>>(d1, a1, (long long)nb * kAct1);
        k_layer_dw<L1><<<gw, 256>>>(spec, kSpecSize, order, d1, g + kOffW1, g + kOffB1);
    }
};

}  // namespace

ProposalNet::~ProposalNet() {
    if (w) cudaFree(w);
    if (bias) cudaFree(bias);
    if (spec) cudaFree(spec);
    if (act) cudaFree(act);
}

bool net_init(ProposalNet& net, const float* weights, int ninst, std::string* err) {
    std::vector<__nv_bfloat16> bf;
    std::vector<float> bias;
    device_layouts(weights, bf, bias);
    if (!net.w && !cuda_ok(cudaMalloc(&net.w, sizeof(__nv_bfloat16) * kBfAll), err, "net weights")) return false;
    if (!net.bias && !cuda_ok(cudaMalloc(&net.bias, sizeof(float) * kBiasAll), err, "net bias")) return false;
    if (net.ninst < ninst) {
        if (net.spec) cudaFree(net.spec);
        if (net.act) cudaFree(net.act);
        net.spec = nullptr;
        net.act = nullptr;
        if (!cuda_ok(cudaMalloc(&net.spec, sizeof(float) * (size_t)ninst * kSpecSize), err, "net spec") ||
            !cuda_ok(cudaMalloc(&net.act, sizeof(float) * (size_t)ninst * kActAll), err, "net activations"))
            return false;
        net.ninst = ninst;
    }
    return cuda_ok(cudaMemcpy(net.w, bf.data(), sizeof(__nv_bfloat16) * kBfAll, cudaMemcpyHostToDevice), err, "w") &&
           cuda_ok(cudaMemcpy(net.bias, bias.data(), sizeof(float) * kBiasAll, cudaMemcpyHostToDevice), err, "bias");
}

void net_run(ProposalNet& net, const BatchDev& b, float* scores, cudaStream_t s) {
    k_spectrogram<<<dim3(kSpecT, b.ninst), kSpecF, 0, s>>>(b, net.spec, kSpecSize, 0);
    k_spec_normalise<<<b.ninst, 256, 0, s>>>(net.spec, b.state, b.iter_max, kSpecSize, 0);
    forward_bf16(net.spec, kSpecSize, net.act, static_cast<const __nv_bfloat16*>(net.w), net.bias, scores, b.ninst,
                 b.state, s);
}

void spectrogram(const BatchDev& b, float* out, cudaStream_t s) {
    const long long stride = (long long)b.iter_max * kSpecSize;
    k_spectrogram<<<dim3(kSpecT, b.ninst), kSpecF, 0, s>>>(b, out, stride, 1);
    k_spec_normalise<<<b.ninst, 256, 0, s>>>(out, b.state, b.iter_max, stride, 1);
}

bool read_weights(const char* path, float* weights, std::string* err) {
    FILE* f = fopen(path, "rb");
    if (!f) {
        if (err) *err = "couldNotOpenProposalWeights";
        return false;
    }
    char magic[8];
    int count = 0;
    const bool good = fread(magic, 1, 8, f) == 8 && memcmp(magic, "EMPIPN01", 8) == 0 &&
                      fread(&count, sizeof(int), 1, f) == 1 && count == kNetParams &&
                      fread(weights, sizeof(float), kNetParams, f) == (size_t)kNetParams;
    fclose(f);
    if (!good && err) *err = "invalidProposalWeights";
    return good;
}

bool net_scores(const float* spec, int n, const float* weights, int bf16, float* scores, std::string* err) {
    if (n <= 0) return true;
    Trainer t(err);
    if (!t.init(spec, nullptr, n, n, weights)) return false;
    std::vector<int> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    if (!cuda_ok(cudaMemcpy(t.order, ord.data(), sizeof(int) * n, cudaMemcpyHostToDevice), err, "order")) return false;
    if (bf16) {
        ProposalNet net;
        if (!net_init(net, weights, n, err)) return false;
        forward_bf16(t.spec, kSpecSize, net.act, static_cast<const __nv_bfloat16*>(net.w), net.bias, t.sc, n, nullptr,
                     0);
    } else {
        t.forward(n);
    }
    return cuda_ok(cudaGetLastError(), err, "forward") &&
           cuda_ok(cudaMemcpy(scores, t.sc, sizeof(float) * (size_t)n * kScores, cudaMemcpyDeviceToHost), err,
                   "scores");
}

bool net_gradients(const float* spec, const int* labels, int n, const float* weights, float* grads, float* loss,
                   std::string* err) {
    Trainer t(err);
    if (n <= 0 || !t.init(spec, labels, n, n, weights)) return n > 0 ? false : true;
    std::vector<int> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    if (!cuda_ok(cudaMemcpy(t.order, ord.data(), sizeof(int) * n, cudaMemcpyHostToDevice), err, "order")) return false;
    t.gradients(n);
    return cuda_ok(cudaGetLastError(), err, "gradients") &&
           cuda_ok(cudaMemcpy(grads, t.g, sizeof(float) * kNetParams, cudaMemcpyDeviceToHost), err, "grads") &&
           cuda_ok(cudaMemcpy(loss, t.loss, sizeof(float), cudaMemcpyDeviceToHost), err, "loss");
}

bool net_train(const float* spec, const int* labels, int n, int epochs, int batch, float lr, float momentum,
               unsigned seed, float* weights, float* losses, std::string* err) {
    if (n <= 0 || epochs <= 0 || batch <= 0) {
        if (err) *err = "invalidArgument";
        return false;
    }
    Trainer t(err);
    if (!t.init(spec, labels, n, std::min(batch, n), weights)) return false;
    std::vector<int> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    std::mt19937 rng(seed);
    for (int e = 0; e < epochs; ++e) {
        std::shuffle(ord.begin(), ord.end(), rng);
        double sum = 0.0;
        int steps = 0;
        for (int s0 = 0; s0 < n; s0 += t.cap) {
            const int nb = std::min(t.cap, n - s0);
            if (!cuda_ok(cudaMemcpy(t.order, ord.data() + s0, sizeof(int) * nb, cudaMemcpyHostToDevice), err, "order"))
                return false;
            t.gradients(nb);
            k_sgd<<<grid_for(kNetParams), 256>>>(t.w, t.v, t.g, kNetParams, lr, momentum);
            float l = 0.0f;
            if (!cuda_ok(cudaMemcpy(&l, t.loss, sizeof(float), cudaMemcpyDeviceToHost), err, "train step"))
                return false;
            sum += l;
            ++steps;
        }
        if (losses) losses[e] = (float)(sum / std::max(1, steps));
    }
    return cuda_ok(cudaMemcpy(weights, t.w, sizeof(float) * kNetParams, cudaMemcpyDeviceToHost), err, "weights");
}

}  // namespace empi
