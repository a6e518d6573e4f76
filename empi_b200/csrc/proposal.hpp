// Learned block proposal: residual log-spectrogram, a 4-layer convolutional
// network scoring the 16 x 32 (scale band, time tile) blocks, its BF16
// tensor-core inference and its FP32 training (proposal.cu).
//
// Network (per instance, channels-first):
//   x0 [1][64][128]   log-magnitude spectrogram (64 bins 0..fs/2 x 128 frames),
//                     normalised to zero mean and unit variance
//   x1 [16][64][128]  conv 3x3, stride 1, pad 1, ReLU
//   x2 [32][32][64]   conv 3x3, stride 2, pad 1, ReLU
//   x3 [32][16][32]   conv 3x3, stride 2, pad 1, ReLU
//   s  [16][32]       per time column, a dense map of the 32 x 16 (channel,
//                     frequency) values to the 16 scale bands: the block scores
// 22,256 parameters, stored FP32 in one vector in the order below.
#pragma once

#include <cstddef>
#include <string>

#include <cuda_runtime.h>

namespace empi {

struct BatchDev;

constexpr int kSpecF = 64, kSpecT = 128;
constexpr int kC1 = 16, kC2 = 32, kC3 = 32, kBands = 16;
constexpr int kH1 = 64, kW1n = 128, kH2 = 32, kW2n = 64, kH3 = 16, kW3n = 32;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kC1 * 9, kOffW2 = kOffB1 + kC1, kOffB2 = kOffW2 + kC2 * kC1 * 9,
              kOffW3 = kOffB2 + kC2, kOffB3 = kOffW3 + kC3 * kC2 * 9, kOffW4 = kOffB3 + kC3,
              kOffB4 = kOffW4 + kBands * kC3 * kH3, kNetParams = kOffB4 + kBands;
constexpr int kSpecSize = kSpecF * kSpecT;
constexpr int kAct1 = kC1 * kH1 * kW1n, kAct2 = kC2 * kH2 * kW2n, kAct3 = kC3 * kH3 * kW3n;
constexpr int kScores = kBands * kW3n;  // 512 = 16 bands x 32 tiles

// Device state of the proposer for a batch: BF16 weights (padded GEMM
// layouts), FP32 biases, per-instance spectrograms and activations.
struct ProposalNet {
    void* w = nullptr;        // BF16 weights of the four layers, GEMM layouts
    float* bias = nullptr;    // FP32 biases of the four layers
    float* spec = nullptr;    // [inst][64][128]
    float* act = nullptr;     // [inst][x1 | x2 | x3]
    int ninst = 0;
    ~ProposalNet();
};

// Uploads FP32 weights (kNetParams) for `ninst` instances; false on a CUDA error.
bool net_init(ProposalNet& net, const float* weights, int ninst, std::string* err);
// Spectrogram of every running instance's residual, then the network's block
// scores into scores [inst][512], on stream s.
void net_run(ProposalNet& net, const BatchDev& b, float* scores, cudaStream_t s);
// The normalised log-spectrogram of every instance's residual into
// out [inst][64][128] (training pairs), on stream s.
void spectrogram(const BatchDev& b, float* out, cudaStream_t s);

// Weights file (the proposer's "EMPIPN01" format): 8-byte magic, int32
// parameter count, the FP32 parameters.  false with a camelCase reason.
bool read_weights(const char* path, float* weights, std::string* err);

// Device-side training and checking, host arrays in and out (proposal.cu):
// inference scores of n spectrograms with BF16 tensor cores (bf16 = 1) or in
// FP32 (bf16 = 0).
bool net_scores(const float* spec, int n, const float* weights, int bf16, float* scores, std::string* err);
// mean cross-entropy loss and its gradient over n (spectrogram, block) pairs,
// FP32 forward and backward kernels.
bool net_gradients(const float* spec, const int* labels, int n, const float* weights, float* grads, float* loss,
                   std::string* err);
// SGD with momentum over the pairs: `epochs` passes in minibatches of
// `batch` (order shuffled by `seed`); weights updated in place, the mean loss
// of each epoch written to losses.
bool net_train(const float* spec, const int* labels, int n, int epochs, int batch, float lr, float momentum,
               unsigned seed, float* weights, float* losses, std::string* err);

}  // namespace empi
