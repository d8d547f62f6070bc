// Launch wrappers of the detection kernels (host-callable, defined in k_*.cu).
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "ccnn_common.cuh"
#include "legacy.h"

namespace ccnn {

struct FaceOut {
    int x, y, w, h;
    float score;
    int gender, smile, glasses;  // facial analysis; -1 without it
    float scale;                 // the merged detection's scale, neighbour count and cluster size
    int knn, num_detect;         // (CNNDetector::Detection, cnn_detector_v3.h:186-217)
    int pad;
};

struct ReplayArgs {
    const Candidate* cands;
    const int* n_cand;
    const WinOut* win;     // 4 per candidate: (window 0, stage 2), (0, 3), (1, 2), (1, 3)
    CandResult* results;   // verdict per candidate (written by the replay kernel)
    const LevelDesc* levels;
    int n_levels;
    CascadeConfig cfg;
    // scratch, each sized for the candidate capacity
    Det* D;          // detections in the reference's cpu_detect_rect order
    Det* R;          // reversed + sorted copy
    Det* M;          // first clustering pass
    Det* F;          // second clustering pass
    int* first_dec;  // per candidate: first decisive earlier box (scan test)
    int* survivors;  // per level: candidates surviving the scan
    uint8_t* checked;
    // facial analysis (null when off): per candidate (dropped, gender, smile, glasses), and
    // scratch of 5 x candidate-capacity ints for the attribute medians of merged boxes
    const int4* attr;
    int* fa_scratch;
    // outputs
    int* n_raw;
    FaceOut* faces;
    int face_cap;
    int* n_faces;
    // the first merge's clusters after the min_num_detect filter (the second merge's input) and
    // their count, for callers that merge them again with detections of their own
    Det* m_out;
    int* n_m_out;
};

// the gray kernel instantiation for `ch` channels, with or without the gate features (to find its
// node in a captured graph)
const void* gray_kernel_fn(int ch, bool feat);
// feat (optional): the learned gate's binary16 input features (W/8 x H/8) written by the same launch
cudaError_t launch_gray(const uint8_t* src, int spitch, int w, int h, int ch, float* dst, int dpitch, cudaStream_t st,
                        __half* feat = nullptr);
cudaError_t launch_gray_u8_resized(const uint8_t* src, int spitch, int sw, int sh, float* dst, int dpitch, int dw, int dh,
                                   cudaStream_t st);
cudaError_t launch_resize_f32(const float* src, int spitch, int sw, int sh, float* dst, int dpitch, int dw, int dh, int type,
                              cudaStream_t st);
// learned scale/region gate (gate.cu): octaves predicted, parameter count, per-frame scratch
constexpr int kGK = 4;
constexpr int kGateParams = 8 * 9 + 8 + 8 * 8 * 9 + 8 + kGK * 8 + kGK;  // 700
struct GateScratch {
    int* ambiguous;  // cells with a probability in [thr / 4, thr); the bitmaps follow it
    uint32_t* bits;  // per octave, per cell row: one bit per cell at or above the threshold
    float* prob;     // kGK x (W/16 x H/16) probabilities
    __half* feat;    // W/8 x H/8 binary16 input features
};
// words of the octave row bitmaps for a gw x gh gray frame
int gate_bitmap_words(int gw, int gh);
// the gate network on the frame's gray image, then the stage-1 tile activity of every level
// the cell bitmaps of a gated frame for the stage-1 back kernel
GateCells gate_cells(GateScratch sc, int gw, int gh, float amb_frac, int margin);
// feat_ready: sc.feat already holds the frame's features (the gray launch wrote them); otherwise they
// are computed from `gray` first
// the gate network's parameters as a kernel parameter (read from the constant bank)
struct GateNet {
    float p[kGateParams];
};
cudaError_t launch_gate(const GateNet& net, const float* gray, int gpitch, int gw, int gh, bool feat_ready, const LevelDesc* levels,
                        int n_levels, GateScratch sc, float thr, float amb_frac, int margin, uint8_t* back_on, uint8_t* front_on,
                        cudaStream_t st);
cudaError_t launch_gate_labels(const Candidate* cands, const CandResult* res, const int* ncand, int cap, const LevelDesc* d_levels, int gw, int gh,
                               uint8_t* labels, cudaStream_t st);

// every level image of a frame into the level arena (img_off / img_pitch of each descriptor), for the
// legacy family (the CNTK stage-1 front kernel resamples its tiles itself); blocks of kPyrCols columns x
// kPyrRows rows (pyr_wq column blocks per level row band)
constexpr int kPyrCols = 256, kPyrRows = 8;
cudaError_t launch_pyramid(const LevelDesc* levels, int n_levels, const float* gray, int gpitch, int gw, int gh, float* limg,
                           cudaStream_t st);
// ---- batched form: one persistent launch runs the pyramid and stage 1 of B frames ----
constexpr int kMaxBatch = 16;
// per-frame buffers of the frames of one batch (frame f = entry f); the gray frames share one size
// and pitch
struct BatchFrames {
    const float* gray[kMaxBatch];
    __half* feat[kMaxBatch];  // the learned gate's input features (written by the gray launch), or null
    int gpitch, gw, gh;
    float* s1[kMaxBatch];
    float* resp[kMaxBatch];
    int* counts[kMaxBatch];
    const uint8_t* front_on[kMaxBatch];  // the learned gate's tile activity, or null
    const uint8_t* back_on[kMaxBatch];
    GateCells cells[kMaxBatch];
};
// the work queue of a batch: segments of items, one per (stage, frame), in queue order; the items of
// a stage are its blocks in the per-frame kernels (stage 0 front tiles, stage 1 back tiles)
constexpr int kBatchStages = 2;
struct BatchQueue {
    int n_frames, n_levels, n_chunks;
    float thr;
    int stage_items[kBatchStages];  // items of one frame per stage
    int n_seg, total;
    int seg_stage[kBatchStages * kMaxBatch], seg_frame[kBatchStages * kMaxBatch], seg_first[kBatchStages * kMaxBatch + 1];
    int wait_limit;                 // polls of a dependency before the launch reports an error
};
// builds the queue order: a diagonal wavefront over (stage, frame), so that the back tiles of frame f
// are queued after the front tiles of frame f+1 (their producer is long done)
void build_batch_queue(BatchQueue* q, int n_frames, int n_levels, int n_chunks, int front_items, int back_items, float thr);
// sync: 1 + kBatchStages * n_frames ints, zero before the launch (queue head, finished items per
// (frame, stage)); err: set to 1 when a dependency wait gave up (results of the batch invalid).
// Front items resample their level tiles from the gray frames (the pyramid is never stored); the
// candidate counts must be zero (launch_counts_zero_batch).
cudaError_t launch_stage1_batch(const Stage1W& W, const BatchFrames& F, const BatchQueue& Q, const LevelDesc* d_levels, int* sync, int* err,
                                int grid, cudaStream_t st, int blocks_per_sm);
// levels of a pyramid the persistent stage-1 kernel takes (their first items live in shared memory);
// deeper pyramids run the per-level kernels
constexpr int kMaxBatchLevels = 256;
// resident blocks of the persistent stage-1 kernel per SM (its grid is this times the SM count)
int stage1_batch_blocks_per_sm(int blocks_per_sm);
// the candidate counts of every frame of a batch zeroed, in one launch
cudaError_t launch_counts_zero_batch(const BatchFrames& F, int n_chunks, int n_frames, cudaStream_t st);

// source of one frame of a batch (device memory, 64-byte aligned base and pitch)
struct FrameSrc {
    const uint8_t* data;
    int pitch;
    int pad;
};
cudaError_t launch_gray_batch(const FrameSrc* d_src, int n_frames, int w, int h, int ch, const BatchFrames& F, int dpitch, cudaStream_t st);
// per-frame outputs of the candidate, window and replay stages of a batch
struct BatchCands {
    Candidate* cands[kMaxBatch];
    int* ncand[kMaxBatch];
};
cudaError_t launch_cand_write_batch(const int4* d_chunks, int n_chunks, const LevelDesc* d_levels, const BatchFrames& F, const BatchCands& C,
                                    int n_frames, float thr, int cap, cudaStream_t st);
struct WinBatch {
    const float* gray[kMaxBatch];
    const Candidate* cands[kMaxBatch];
    const int* ncand[kMaxBatch];
    WinOut* out[kMaxBatch];
    int n_frames;
};
cudaError_t launch_window_batch(const WindowNets& N, const WinBatch& B, int gpitch, int gw, int gh, const LevelDesc* levels,
                                const CascadeConfig& cfg, int grid, cudaStream_t st, int ctas_per_sm = 4);
// the replay of every frame of a batch: block f runs args[f] (device memory)
cudaError_t launch_replay_batch(const ReplayArgs* d_args, int n_frames, cudaStream_t st);

// register budget of the stage-1 kernels: resident 256-thread blocks per SM (3 or 4), a schedule knob
struct Stage1Sched {
    int front_blocks_per_sm = 3;
    int back_blocks_per_sm = 4;
};
// the frame's gray image as the stage-1 front kernel resamples each level tile from it; p == nullptr:
// the level images are stored (limg + img_off) and read instead
struct GrayRef {
    const float* p;
    int pitch, w, h;
};
// stage-1 net over all levels; `levels` is a HOST array (the descriptors travel as kernel
// parameters); level tiles resampled from `gray`, or read from limg + img_off when gray.p is null
// counts (optional, zeroed by the caller): per candidate-scan chunk, responses > thr
// cells (optional): the gate's cell bitmaps; a response above thr whose window centre has no likely
// cell within cells.margin cells of it (in its level's octave) is written below every threshold
cudaError_t launch_stage1(const Stage1W& W, const LevelDesc* levels, int n_levels, const float* limg, float* s1, float* resp,
                          cudaStream_t st, int* counts = nullptr, float thr = 0.f, const uint8_t* front_on = nullptr,
                          const uint8_t* back_on = nullptr, GateCells cells = GateCells{}, Stage1Sched sched = Stage1Sched{},
                          GrayRef gray = GrayRef{});
// front_on / back_on (optional): per-tile activity from the gate; inactive back tiles write
// responses below every threshold
cudaError_t launch_stage1_front(const Stage1W& W, const LevelDesc* levels, int n_levels, const float* limg, float* s1, cudaStream_t st,
                                const uint8_t* front_on = nullptr, Stage1Sched sched = Stage1Sched{}, GrayRef gray = GrayRef{},
                                GateCells cells = GateCells{});
// dynamic shared memory of the stage-1 back kernel (set once per device before any launch)
cudaError_t stage1_setup();
cudaError_t launch_stage1_back(const Stage1W& W, const LevelDesc* levels, int n_levels, const float* s1, float* resp, cudaStream_t st,
                               int* counts = nullptr, float thr = 0.f, const uint8_t* back_on = nullptr, GateCells cells = GateCells{},
                               Stage1Sched sched = Stage1Sched{});
cudaError_t launch_cand_write(const int4* d_chunks, int n_chunks, const LevelDesc* d_levels, const float* resp, float thr,
                              const int* counts, Candidate* out, int* n_out, int cap, cudaStream_t st);
// lg (optional): the legacy networks (device memory, [1] stage 2, [2] stage 3) replace N
// ctas_per_sm: resident blocks a SM the grid was sized for (1-6); 2 or fewer selects the
// 128-register build, 5 and 6 the 48- and 40-register ones
cudaError_t window_setup();
cudaError_t launch_window(const WindowNets& N, const float* gray, int gpitch, int gw, int gh, const Candidate* cands, const int* n_cand,
                          const LevelDesc* levels, WinOut* out, const CascadeConfig& cfg, int grid, cudaStream_t st,
                          const LegacyNet* lg = nullptr, int ctas_per_sm = 4);
// one legacy (format 1.0) network on a w x h image (pitch floats): scratch holds its pooled L1 and
// L2 maps; counts (optional) gets each scan chunk's responses above thr
cudaError_t launch_legacy_forward(const LegacyNet* d_net, const LegacyNet& h_net, const float* img, int pitch, int w, int h, float* scratch,
                                  float* resp, cudaStream_t st, int* counts, int chunk_base, float thr);
int window_smem_bytes();
// facial analysis: dynamic shared memory attribute (once per device) and the landmark kernel
cudaError_t facial_setup();
cudaError_t launch_facial(const LandmarkNet* d_net, const float* gray, int gpitch, int gw, int gh, const Candidate* cands,
                          const int* n_cand, const LevelDesc* levels, const WinOut* win, const CascadeConfig& cfg, int4* attr, int grid,
                          cudaStream_t st);
// dynamic shared memory of the replay kernel (set once per device before any launch)
constexpr int kReplaySmemBytes = 200 * 1024;
cudaError_t replay_setup();
cudaError_t launch_replay(const ReplayArgs& a, cudaStream_t st);
// the replay kernel's block-wide sort on n keys (synchronous; for tests): perm[i] = input index of
// the i-th key after sorting by scale, descending, in libstdc++ std::sort's order of ties
cudaError_t sort_permutation_device(const float* scales, int n, int* perm);
// CNNDetector::Detect with detections already in the caller's vector (cnn_detector_v3.cpp:2753-2806):
// [prior, new clusters] through the min_num_detect filter (applied to the priors here; the clusters
// come filtered) and Merger(0.2, del), then the optional rescale; scratch holds 2 * (n_prior + n_new)
// Det and as many bytes. The result goes to out / *n_out.
cudaError_t launch_prior_merge(const Det* prior, int n_prior, const Det* clusters, const int* n_clusters, const CascadeConfig& cfg, Det* scratch,
                               uint8_t* checked, Det* out, int* n_out, cudaStream_t st);
// CNNDetector::NMS = Merger(detections, rect, 0.5) (cnn_detector_v3.cpp:2814-2936) of n boxes
cudaError_t launch_nms(const Det* in, int n, uint8_t* checked, Det* out, int* n_out, cudaStream_t st);

}  // namespace ccnn
