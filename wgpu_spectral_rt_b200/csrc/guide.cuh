// guide.cuh — neural path guiding: network layout, device buffers and the
// launch interface of guide.cu.
//
// Network (no reference counterpart; defined by this project): 10 inputs
// (position in the scene bounds, shading normal, outgoing direction,
// wavelength, each mapped to [0, 1]) -> frequency encoding (sin, cos of
// 2^k * pi * x, k = 0..5: 120 features, zero-padded to 128) -> 4 hidden
// layers of 64 ReLU units -> 48 linear outputs: 8 von Mises-Fisher lobes
// (direction 3, log kappa 1, mixture logit 1) and the selection logit of
// the one-sample mixture of guide and BSDF sampling.  BF16 weights on the
// tensor cores with FP32 accumulation; FP32 master weights and Adam state.
#pragma once

#include <cuda_bf16.h>

#include "device_common.cuh"

namespace srt {

constexpr int G_IN = 10;
constexpr int G_ENC = 128;
constexpr int G_HID = 64;
constexpr int G_OUT = 48;
constexpr int G_LOBES = 8;
constexpr int G_LAYERS = 5;
constexpr float G_KAPPA_LO = -4.0f, G_KAPPA_HI = 7.0f;
constexpr float G_SEL_LO = 0.05f, G_SEL_SPAN = 0.85f;

// layer l: in -> out
__host__ __device__ constexpr int g_in(int l) { return l == 0 ? G_ENC : G_HID; }
__host__ __device__ constexpr int g_out(int l) { return l == 4 ? G_OUT : G_HID; }
// flat parameter offsets: W0 b0 W1 b1 ... (W [out][in] row-major)
__host__ __device__ constexpr int g_woff(int l) {
    return l == 0 ? 0 : (G_ENC + 1) * G_HID + (l - 1) * (G_HID + 1) * G_HID;
}
__host__ __device__ constexpr int g_boff(int l) { return g_woff(l) + g_in(l) * g_out(l); }
constexpr int G_NPARAMS = g_boff(4) + G_OUT;  // 23856
static_assert(G_NPARAMS == 23856 && g_boff(3) + G_HID == g_woff(4), "guide parameter layout");

// Shared-memory rows are padded by 8 bf16 so that the 8 rows a fragment
// load touches fall in different banks.
__host__ __device__ constexpr int g_pad(int n) { return n + 8; }

struct GuideNet {
    float* master;          // G_NPARAMS fp32
    __nv_bfloat16* wbf;     // bf16 weights, same flat offsets (biases unused)
    float* adam_m;          // G_NPARAMS
    float* adam_v;          // G_NPARAMS
    float* grad;            // G_NPARAMS fp32 accumulators (zeroed by the Adam step)
};

// Per-bounce buffers of the diffuse vertices whose continuation the guide samples.
struct GuideVerts {
    float4* p;     // hit point xyz, hero wavelength
    float4* n;     // face-forwarded shading normal
    float4* wo;    // outgoing direction (towards the previous vertex)
    float4* spec;  // reflectance spectrum at the 4 wavelengths
    uint32_t* id;  // path id
};

// Training samples recorded during a frame (capacity G_REC_CAP).
struct GuideRecords {
    float4* x0;    // inputs 0..3
    float4* x1;    // inputs 4..7
    float4* x2;    // inputs 8..9, unused
    float4* w;     // sampled direction xyz, pdf it was sampled with
    float4* b;     // BSDF pdf, f*cos (scalar), unused, unused
    float4* thr;   // throughput after the vertex
    float4* rad;   // path radiance at the start of the next vertex (NaN: not reached)
    uint32_t* pid; // path id
    float* weight; // training weight F / p_sample
    // training activations and deltas (bf16, [sample][feature])
    __nv_bfloat16* act;    // G_REC_CAP x (128 + 4 x 64)
    __nv_bfloat16* delta;  // G_REC_CAP x (4 x 64 + 48)
};
constexpr uint32_t G_REC_CAP = 1u << 18;
constexpr uint32_t G_BATCH_DEFAULT = 1u << 16;  // training samples per frame
constexpr int G_ACT_STRIDE = G_ENC + 4 * G_HID;    // 384
constexpr int G_DELTA_STRIDE = 4 * G_HID + G_OUT;  // 304
__host__ __device__ constexpr int g_act_off(int l) { return l < 0 ? 0 : G_ENC + l * G_HID; }  // input of layer l+1
__host__ __device__ constexpr int g_delta_off(int l) { return l * G_HID; }

// Device-side counters of the guide (in the frame counters block).
struct GuideCounters {
    uint32_t verts[32];      // guided vertices per bounce
    uint32_t records;        // training samples recorded this frame
    uint32_t candidates;     // diffuse vertices eligible for recording
    uint32_t threshold;      // recording threshold (of 65536) for the next frame
    uint32_t adam_step;      // Adam steps taken
    float weight_sum;        // sum of training weights this frame
    float pad2[3];
};

struct GuideArgs {
    GuideNet net;
    GuideVerts gv;
    GuideRecords rec;
    GuideCounters* gc;
    int train;               // run a training step after each frame
    float lr;
    uint32_t batch;          // training samples recorded per frame (<= G_REC_CAP)
    uint32_t steps;          // Adam steps per frame, each on a consecutive 1/steps of the records
    int tc;                  // inference on tcgen05 / tensor memory (else mma.sync)
    int tc_train;            // training step on tcgen05 (k_guide_train_tc; else mma.sync + split-K)
    uint32_t* err;           // device error word (an MMA wait that gave up), may be null
};
static_assert(G_NPARAMS % 8 == 0 && g_woff(1) % 8 == 0 && g_woff(2) % 8 == 0 && g_woff(3) % 8 == 0 &&
                  g_woff(4) % 8 == 0,
              "bf16 weight blocks start on 16-byte boundaries");

// Launchers (guide.cu); each returns the number of kernels it launched.
struct FrameArgs;
cudaError_t guide_configure();  // raises the dynamic shared-memory limits once per device
int launch_guide_infer(const FrameArgs& a, uint32_t bounce, cudaStream_t st);
int launch_guide_train(const FrameArgs& a, cudaStream_t st);
// The two halves of launch_guide_train: the training weights of the frame's
// records (reads the frame's path radiance; before the next frame's camera
// rays), then the Adam steps and the frame-end bookkeeping (before the next
// frame's shading).
int launch_guide_targets(const FrameArgs& a, cudaStream_t st);
int launch_guide_steps(const FrameArgs& a, cudaStream_t st);
// Many renderers at once (device array of their frame arguments, the batched
// renderer): the guided vertices of one bounce in one persistent tcgen05
// launch (fetch: a zeroed chunk counter), and one training step of every
// item (those with train set) in five grouped launches.
int launch_guide_infer_multi(const FrameArgs* items, int n_items, uint32_t bounce, uint32_t* fetch, int sm_count,
                             cudaStream_t st);
int launch_guide_train_multi(const FrameArgs* items, int n_items, uint32_t max_steps, int sm_count,
                             cudaStream_t st);
// tc: the tcgen05 kernel (err: device error word for an MMA wait that gave up).
int launch_guide_test_forward(const GuideNet& net, const float* x, uint32_t n, float* y, int tc, uint32_t* err,
                              cudaStream_t st);
// tc: the mixture functions of the tcgen05 inference kernel (else the mma.sync kernel's lane-pair form)
int launch_guide_test_mixture(const float* raw, const float* omega, const float* u, uint32_t n, float* out, int tc,
                              cudaStream_t st);
// phase 0: forward + backward + weight gradients of gc->records records
// (gc->weight_sum set by the caller; g.steps = 1); phase 1: one Adam step.
int launch_guide_test_train(const GuideArgs& g, int phase, cudaStream_t st);
// One block waiting on an mbarrier that never completes, `polls` polls at most.
int launch_test_wait_timeout(uint32_t polls, uint32_t* err, cudaStream_t st);

// Host side: deterministic default weights (G_NPARAMS floats), device
// buffers for n_verts guided vertices per bounce and G_REC_CAP records, and
// the upload of FP32 weights (+ their bf16 copies) and Adam state.
void guide_default_params(uint64_t seed, float* out);
cudaError_t guide_alloc(GuideArgs& g, size_t n_verts);
void guide_free(GuideArgs& g);
// The trainable state (FP32 and bf16 weights, Adam moments, counters) to or
// from a device buffer of guide_state_bytes() (stream-ordered copies).
size_t guide_state_bytes();
cudaError_t guide_state_copy(GuideArgs& g, void* buf, bool save, cudaStream_t st);
cudaError_t guide_upload(GuideArgs& g, const float* params, const float* adam_m, const float* adam_v,
                         uint32_t adam_step);

}  // namespace srt
