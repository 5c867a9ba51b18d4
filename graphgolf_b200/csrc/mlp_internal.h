// mlp_internal.h -- the proposal filter's network object and the enqueue
// helpers the annealing engine calls (all on a caller-given stream, usable
// inside a stream capture).  Not part of the public C ABI.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace ggb {
namespace mlp {

constexpr int kFeatures = 32;
constexpr int kHidden = 256;
constexpr int kMaxTrainRows = 256;
// Packed FP32 parameters: W1 [256][32], b1 [256], W2 [256][256] (row n holds
// the weights into unit n), b2 [256], w3 [256], b3 [1].
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kHidden * kFeatures;
constexpr int kOffW2 = kOffB1 + kHidden;
constexpr int kOffB2 = kOffW2 + kHidden * kHidden;
constexpr int kOffW3 = kOffB2 + kHidden;
constexpr int kOffB3 = kOffW3 + kHidden;
constexpr int kParams = kOffB3 + 1;

struct AdamHyper {
  float lr, beta1, beta2, eps;
};

}  // namespace mlp
}  // namespace ggb

struct ggb_mlp {
  int max_rows = 0;
  ggb::mlp::AdamHyper hyper{};
  float* p = nullptr;          // FP32 master parameters
  float* g = nullptr;          // gradients of the last backward
  float* m1 = nullptr;         // Adam moments
  float* m2 = nullptr;
  int* step = nullptr;         // Adam step count (device)
  __nv_bfloat16* W1b = nullptr;    // [256][32]
  __nv_bfloat16* W2b = nullptr;    // [256][256]
  __nv_bfloat16* W2tb = nullptr;   // W2 transposed
  // W1 and W2 in the tensor cores' shared-memory operand layout (K-major,
  // no swizzle: 8-row x 16-byte core matrices), staged by one bulk copy each
  __nv_bfloat16* W1u = nullptr;    // [256][32] tiled
  __nv_bfloat16* W2u = nullptr;    // [256][256] tiled
  // activations and workspaces
  __nv_bfloat16* H1 = nullptr;     // [max_rows][256]
  float* H2 = nullptr;             // [max_rows][256]
  float* Z2 = nullptr;             // [max_rows][256]
  float* y_train = nullptr;        // [kMaxTrainRows]
  __nv_bfloat16* dZ2 = nullptr;    // [kMaxTrainRows][256]
  __nv_bfloat16* dZ2t = nullptr;
  __nv_bfloat16* H1t = nullptr;
  __nv_bfloat16* dZ1 = nullptr;
  float* dZ1f = nullptr;
  __nv_bfloat16* dZ1t = nullptr;
  __nv_bfloat16* Xt = nullptr;     // [32][kMaxTrainRows]
  __nv_bfloat16* Xs = nullptr;     // gathered training rows [kMaxTrainRows][32]
  float* loss = nullptr;
  // host-entry staging
  __nv_bfloat16* X = nullptr;      // [max_rows][32]
  float* y = nullptr;              // [max_rows]
  float* t = nullptr;              // [kMaxTrainRows]
};

namespace ggb {

// y[0..rows) = network(X rows); rows % 16 == 0.  keep_z keeps the second
// layer's pre-activations for a backward pass.
int mlp_forward(ggb_mlp* m, const __nv_bfloat16* X, int rows, float* y, cudaStream_t st, bool keep_z);
// Gradients of the mean squared error over B rows (B % 16 == 0, B <= 256).
int mlp_backward(ggb_mlp* m, const __nv_bfloat16* Xs, const float* t, int B, cudaStream_t st);
// One Adam step with the last gradients.
int mlp_adam(ggb_mlp* m, cudaStream_t st);
// Gathers rows idx[0..B) of X, then backward + Adam on them with targets t.
int mlp_train_rows(ggb_mlp* m, const __nv_bfloat16* X, const int* idx, const float* t, int B, cudaStream_t st);
// The training state (FP32 parameters, both Adam moments, the Adam step) as
// host bytes: its size, a copy out and a copy in (which also refreshes every
// BF16 copy of the weights).  Synchronous.
size_t mlp_state_bytes();
int mlp_save_state(ggb_mlp* m, void* host);
int mlp_load_state(ggb_mlp* m, const void* host);

}  // namespace ggb
