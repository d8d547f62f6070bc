// Host runtime of the detection path: configuration, pyramid planning, device buffers,
// CUDA-graph capture of the per-frame kernel chain, result download.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/ccnn.h"
#include "../../include/ccnn_inspect.h"
#include "../../include/ccnn_gate.h"
#include "../../include/ccnn_cnn.h"
#include "legacy.h"
#include "kernels.h"

namespace ccnn {

// One pyramid plan: everything that depends on the frame size and the level count in force.
struct Plan {
    int in_w = 0, in_h = 0, ch = 0;  // input frame
    size_t in_pitch = 0;             // bytes per row of the frame in the slot's input buffer (packed to 64)
    int gw = 0, gh = 0;              // gray image (after the optional 8-bit downscale)
    bool downscale = false;
    int n_levels = 0;                // processed levels scl = 0 .. n_levels-1
    std::vector<LevelDesc> levels;
    std::vector<int4> chunks;        // candidate-scan chunks in visiting order
    int k1_tiles = 0, k2_tiles = 0;
    long long s1_floats = 0, resp_floats = 0, img_floats = 0;
    LevelDesc* d_levels = nullptr;
    int4* d_chunks = nullptr;
};

// Device buffers and stream of one in-flight frame.
struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    uint8_t* d_in = nullptr;
    size_t in_pitch = 0;
    float* d_gray = nullptr;
    int gray_pitch = 0;  // floats
    float* d_limg = nullptr;  // level arena: every level image of the frame (legacy family only)
    float* d_s1 = nullptr;
    float* d_resp = nullptr;
    int* d_counts = nullptr;
    Candidate* d_cands = nullptr;
    int* d_ncand = nullptr;
    CandResult* d_results = nullptr;
    WinOut* d_win = nullptr;
    Det *D = nullptr, *R = nullptr, *M = nullptr, *F = nullptr;
    int* first_dec = nullptr;
    int* survivors = nullptr;
    uint8_t* checked = nullptr;
    int* d_nraw = nullptr;
    FaceOut* d_faces = nullptr;
    int* d_nfaces = nullptr;
    int* h_nfaces = nullptr;   // pinned: face count, then the single-launch stage 1's error flag
    int* d_sync1 = nullptr;    // single-launch stage 1: queue head, finished items per stage, error flag
    FaceOut* h_faces = nullptr;  // pinned, kHostFaces entries
    GateScratch gate{};          // learned gate: features, activations, probabilities (when enabled)
    uint8_t* d_front_on = nullptr;  // learned gate: stage-1 tile activity
    uint8_t* d_back_on = nullptr;
    int4* d_attr = nullptr;      // facial analysis: per candidate (dropped, gender, smile, glasses)
    int* d_fa = nullptr;         // facial analysis: replay scratch (5 x candidate capacity)
    Det* d_mk = nullptr;         // the first merge's filtered clusters of the last frame
    int* d_nmk = nullptr;
    cudaGraphExec_t exec = nullptr;
    const Plan* exec_plan = nullptr;
    cudaGraph_t graph = nullptr;          // kept while `exec` lives: its gray-kernel node is updated per frame
    cudaGraphNode_t gray_node = nullptr;  // the gray conversion, retargeted at a device frame read in place
    cudaKernelNodeParams gray_kp{};
    __half* gray_feat = nullptr;          // the gate features the captured gray node writes, or null
    bool gray_in_place = false;           // the node currently reads the caller's frame
    bool last_in_place = false;           // the last frame was not copied into d_in
    const Plan* last_plan = nullptr;  // plan of the last frame run on this slot
    std::vector<FaceOut> h_extra;     // faces beyond the pinned buffer's kHostFaces
};

// A batch context: B consecutive frame slots whose frames run as one captured graph (batched gray,
// one persistent launch for the pyramid and stage 1 of every frame, batched candidate write, windows
// and replay), with the group's sources and results in its own buffers.
struct BatchCtx {
    int first_slot = 0;
    cudaEvent_t done = nullptr;
    int* d_sync = nullptr;        // queue head, finished items per (frame, stage), error flag
    ReplayArgs* d_rargs = nullptr;
    FrameSrc* d_src = nullptr;
    FrameSrc* h_src = nullptr;    // pinned
    FaceOut* d_faces = nullptr;   // B x face capacity
    int* d_nf = nullptr;          // B face counts
    FaceOut* h_faces = nullptr;   // pinned, B x kGraphFaces
    int* h_nf = nullptr;          // pinned, B face counts and the error flag
    cudaGraphExec_t exec = nullptr;
    const Plan* exec_plan = nullptr;
    bool exec_gated = false;
    int pending_first = -1;       // index in the caller's image array of the frames in flight
    std::vector<FaceOut> h_extra;
};

class Detector {
   public:
    static constexpr int kSlots = 8;
    static constexpr int kHostFaces = 1024;
    static constexpr int kGraphFaces = 64;  // faces each frame's graph downloads; more are fetched on demand

    Detector() = default;
    ~Detector();

    // n_slots: frames in flight (each slot owns a stream, buffers and a captured graph);
    // colour_input: start in the state the reference reaches after its first colour frame
    // (gray_image_only off), so that colour frames never re-initialise the detector
    ccnn_status create(const ccnn_params& p, const char* const* model_paths, int n_slots = kSlots, bool colour_input = false);
    ccnn_status detect(const ccnn_image& img, bool device_input, cudaStream_t user_stream, ccnn_face* faces, int cap, int* n);

    // The internal CNNDetector class (cnn_detector_v3.h:82-453): its Param + AdvancedParam instead of
    // FaceDetector::Param, raw Detection results, the caller's prior detections, NMS.
    ccnn_status create_cnn(const ccnn_cnn_param& p, const ccnn_cnn_advanced_param& ap, const char* const* model_paths);
    ccnn_status detect_cnn(const ccnn_image& img, const ccnn_detection* prior, int n_prior, ccnn_detection* out, int cap, int* n);
    ccnn_status nms(const ccnn_detection* rect, int n_rect, ccnn_detection* out, int cap, int* n_out);
    ccnn_status get_cnn_params(ccnn_cnn_param* p, ccnn_cnn_advanced_param* ap);
    ccnn_status set_cnn_params(const ccnn_cnn_param* p, const ccnn_cnn_advanced_param* ap);
    ccnn_status detect_batch(const ccnn_image* imgs, int n_img, bool device_input, ccnn_face* faces, int cap_per, int* n_faces,
                             float* gpu_ms);
    ccnn_status profile(int iters, float* ms, int n_ms);
    // learned scale/region gate: parameters (kGateParams floats), probability threshold, and the
    // fraction of ambiguous cells above which a frame falls back to the full scan
    ccnn_status gate_set(const float* params, int n, float threshold, float fallback_fraction);
    ccnn_status gate_disable();
    // schedule knobs an autotuner sets: frames in flight and resident stage-2/3 blocks per SM
    // (0 keeps the current value); the device state is rebuilt
    ccnn_status set_schedule(int frame_slots, int window_ctas_per_sm, int front_bpsm = 0, int back_bpsm = 0, int batch_frames = -1,
                             int batch_bpsm = 0);
    void get_schedule(int* frame_slots, int* window_ctas_per_sm, int* front_bpsm = nullptr, int* back_bpsm = nullptr,
                      int* batch_frames = nullptr, int* batch_bpsm = nullptr) const;
    // training labels of the last frame (slot 0): uint8 [4][gh/16][gw/16], device memory
    ccnn_status gate_labels(uint8_t* d_labels, cudaStream_t st);
    // stage-1 tiles the gate let run in the last frame (slot 0), of all, and whether it fell back
    ccnn_status gate_stats(int* front_run, int* front_total, int* back_run, int* back_total, int* fallback);
    ccnn_status gate_probabilities(float* out, int cap, int* n);
    ccnn_status gate_set_margin(int pixels);

    // Non-blocking use of one slot by a single scheduling thread (the serving loop): launch a
    // host frame on slot k, test for completion, fetch the faces. Frames must have the size the
    // detector was created for.
    int n_slots() const { return (int)slots_.size(); }
    ccnn_status launch(int k, const ccnn_image& img);
    bool slot_done(int k);
    ccnn_status fetch(int k, ccnn_face* faces, int cap, int* n);
    // device bytes held by the frame slots
    size_t slot_bytes() const;
    long long limg_floats() const;
    // the device bytes create() would allocate for these arguments, computed on the host without
    // touching the device (so that a caller can make room before allocating)
    static ccnn_status estimate_bytes(const ccnn_params& p, const char* const* model_paths, int n_slots, bool colour_input,
                                      bool with_gate, size_t* bytes);

    ccnn_status get_gray_device(const float** data, int* cols, int* rows, size_t* step);
    ccnn_status get_gray_host(float* out, int cap, int* cols, int* rows);
    ccnn_status get_params(ccnn_params* out);
    ccnn_status set_params(const ccnn_params& p);
    ccnn_status set_max_image_size(int w, int h);
    ccnn_status set_min_object_height(int v);
    ccnn_status set_max_object_height(int v);
    ccnn_status set_num_threads(int v);

    ccnn_status stage1_forward(const float* d_img, int w, int h, size_t step, float* d_resp, int cap, int* rw, int* rh, cudaStream_t st);
    ccnn_status inspect_levels(ccnn_level_info* out, int cap, int* n);
    ccnn_status inspect_response(int level, float* out, int cap);
    ccnn_status inspect_candidates(ccnn_candidate* out, int cap, int* n);
    ccnn_status inspect_raw(ccnn_detection* out, int cap, int* n);

   private:
    // configuration (FaceDetector::Param + the AdvancedParam the API derives from it)
    ccnn_params api_{};
    // created through the CNNDetector API: its Param and AdvancedParam as given (the precision
    // rules are applied on top at every initialisation)
    bool has_cnn_ = false;
    ccnn_cnn_param cnn_p_{};
    ccnn_cnn_advanced_param cnn_ap_{};
    void cnn_to_api();
    int device_ = 0;
    bool gray_image_only_ = true;
    int type_check_ = 2, min_num_detect_ = 1;
    bool adapt_min_neighbors_ = false, drop_detect_ = true, detect_enabled_ = true, merger_detect_ = true;
    bool equalize_ = true, reflection_ = true, double_check_ = true;

    // models
    std::string model_paths_[3];
    Stage1W w1_{};
    std::unique_ptr<WindowNets> wn_;
    LandmarkNet* d_lnet_ = nullptr;  // facial-analysis network (device memory), when enabled
    std::unique_ptr<LandmarkNet> h_lnet_;  // its host copy
    // legacy model family (format 1.0): the three networks on the host and in device memory
    bool legacy_ = false;
    std::unique_ptr<LegacyNet[]> h_lg_;
    LegacyNet* d_lg_ = nullptr;
    ccnn_status enqueue_legacy_stage1(Slot& s, const Plan& p);
    int window_ctas_per_sm_ = 4;     // persistent stage-2/3 grid: this many blocks per SM
    Stage1Sched s1_sched_{};         // stage-1 register budgets
    int batch_frames_ = 0;           // frames per batched launch (0: every frame its own graph; 1: every frame
                                     // its own graph with the pyramid and stage 1 in one persistent launch)
    bool single_launch_stage1() const;
    int batch_bpsm_ = 3;             // resident blocks per SM (grid) of the persistent stage-1 kernel
    std::vector<BatchCtx> batches_;
    int sm_count_ = 0;
    ccnn_status alloc_batches();
    void free_batches();
    ccnn_status enqueue_batch_kernels(BatchCtx& c, const Plan& p, int B);
    ccnn_status launch_batch(BatchCtx& c, const Plan& p, const ccnn_image* imgs, int B, bool device_input);
    ccnn_status collect_batch(BatchCtx& c, int B, ccnn_face* faces, int cap_per, int* n_faces, ccnn_status* worst);
    bool batch_usable(const Plan& p) const;
    GateNet gate_net_{};             // learned gate parameters (passed to the inference kernel by value)
    bool gate_on_ = false;
    float gate_thr_ = 0.5f, gate_amb_frac_ = 0.25f;
    int gate_margin_ = 16;           // pixels around a candidate's window centre the gate searches
    std::vector<float> gate_params_;
    ccnn_status alloc_gate(Slot& s);
    int pat_w_ = kPatW, pat_h_ = kPatH;     // stage-1 window
    int ext_w_ = kWinW, ext_h_ = kWinH;     // smallest level processed

    // initialised state (CNNDetector::Init)
    bool inited_ = false;
    int max_w_ = 0, max_h_ = 0;
    std::vector<float> scales_;
    bool input_downscale_ = false;
    float input_scale_ = 0.f;
    int num_scales_ = 0;

    CascadeConfig cfg_{};
    std::vector<Slot> slots_;
    long long cand_cap_ = 0, s1_cap_ = 0, resp_cap_ = 0, img_cap_ = 0;
    int k1_cap_ = 0, k2_cap_ = 0;
    int chunk_cap_ = 0;
    int window_grid_ = 0;
    int facial_grid_ = 0;
    std::map<std::tuple<int, int, int, int>, std::unique_ptr<Plan>> plans_;
    std::mutex mu_;
    // orders device frames after the caller's work on the legacy default stream
    cudaEvent_t order_ev_ = nullptr;
    int init_gen_ = 0;  // counts initialisations (each recreates the slot streams)

    ccnn_status init();
    // the host half of init(): models, scales, plan capacities; touches no device
    ccnn_status init_host();
    // the slot streams wait for the work queued so far on `user_stream`, or on the legacy default
    // stream when it is null (the stream a caller without one of its own, torch included, writes on)
    ccnn_status order_after(cudaStream_t user_stream, int n_slots);
    void clear();
    ccnn_status alloc_slot(Slot& s);
    void free_slot(Slot& s);
    ccnn_status plan_for(int w, int h, int ch, const Plan** out);
    ccnn_status build_plan(int w, int h, int ch, int num_scales, Plan* p);
    ccnn_status enqueue(Slot& s, const Plan& p, const ccnn_image& img, bool device_input, cudaStream_t copy_stream);
    ccnn_status enqueue_kernels(Slot& s, const Plan& p);
    ccnn_status prepare_frame(const ccnn_image& img, const Plan** plan, bool* empty);
    ccnn_status collect(Slot& s, ccnn_face* faces, int cap, int* n);
    ccnn_status collect_raw(Slot& s, int cap, int* n, const FaceOut** src);
    ReplayArgs replay_args(Slot& s, const Plan& p) const;
    ccnn_status apply_precision();
};

bool compute_scales(const ccnn_params& p, bool gray_only, int pat_h, int max_h, std::vector<float>* scales, bool* downscale,
                    float* input_scale);
void set_error(const std::string& msg);
ccnn_status cuda_status(cudaError_t e, const char* what);

}  // namespace ccnn
