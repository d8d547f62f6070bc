// Host runtime of the B200 detection path.
//
// Mirrors the reference's CNNDetector lifecycle (src/CNNObjectDetector/cnn_detector_v3.cpp):
// Init (:907-985) with the precision rules (:922-963) and InitScales (:289-346); Detect
// (:2483-2813) with its re-initialisation rules (frame larger than max_image_size :2499-2513,
// multi-channel frame while gray_image_only :2531-2546) and the level-count state num_scales
// that RunCPUDetect lowers when a level is smaller than the stage-2/3 window (:2083-2088).
// The parameters are FaceDetector::Param converted as paramConverter does
// (CompactCNNLibAPI_v2.cpp:280-329).
//
// Per frame the device runs: gray conversion -> stage-1 front (all levels) -> stage-1 back (all
// levels) -> candidate count -> candidate write -> stage-2/3 windows -> replay/sort/merge, plus
// the download of the face count and the first faces. The chain is captured once per
// (slot, pyramid plan) as a CUDA graph and replayed; only the frame upload is issued per call.
#include "detector.h"
#include "model.h"

#include <algorithm>
#include <cstdint>
#include <cmath>
#include <cstring>

namespace ccnn {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error_cstr() { return g_last_error.c_str(); }

ccnn_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CCNN_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return CCNN_ERR_OOM;
    return CCNN_ERR_CUDA;
}

#define CCNN_CUDA(call)                                         \
    do {                                                        \
        ccnn_status _s = cuda_status((call), #call);            \
        if (_s != CCNN_OK) return _s;                           \
    } while (0)

namespace {
inline long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }
// Size * float with truncation (type.h:200-203)
inline void size_scale(int w, int h, float s, int* ow, int* oh) {
    *ow = (int)((float)w * s);
    *oh = (int)((float)h * s);
}
}  // namespace

// InitScales (cnn_detector_v3.cpp:289-346): scales from max_scale = min(3, 27 / min face) down
// to min_scale = 27 / max face (or / max image height) by repeated division by the factor. With
// gray-only input and max_scale < 0.8 the frame itself is shrunk by max_scale and the pyramid
// starts at 1.
bool compute_scales(const ccnn_params& p, bool gray_only, int pat_h, int max_h, std::vector<float>* scales, bool* downscale,
                    float* input_scale) {
    scales->clear();
    *downscale = false;
    *input_scale = 0.f;
    float max_scale = 1.f;
    if (p.min_face_height > 0) {
        max_scale = (float)pat_h / (float)p.min_face_height;
        max_scale = 3.f > max_scale ? max_scale : 3.f;
        if (gray_only && max_scale < 0.8f) {
            *downscale = true;
            *input_scale = max_scale;
            max_scale = 1.f;
        }
    }
    float min_scale = p.max_face_height > 0 ? (float)pat_h / (float)p.max_face_height : (float)pat_h / (float)max_h;
    min_scale = max_scale > min_scale ? min_scale : max_scale;
    const float sf = p.scale_factor < 1.f ? 1.1f : p.scale_factor;
    float scale = max_scale;
    if (sf != 1.f) {
        while (scale > min_scale) {
            scales->push_back(scale);
            scale /= sf;
        }
    } else {
        scales->push_back(scale);
    }
    return !scales->empty();
}

Detector::~Detector() {
    clear();
    if (order_ev_) cudaEventDestroy(order_ev_);
    if (d_lnet_) cudaFree(d_lnet_);
    if (d_lg_) cudaFree(d_lg_);
}

void Detector::free_slot(Slot& s) {
    if (s.exec) cudaGraphExecDestroy(s.exec);
    if (s.graph) cudaGraphDestroy(s.graph);
    cudaFree(s.d_in);
    cudaFree(s.d_gray);
    cudaFree(s.d_limg);
    cudaFree(s.d_attr);
    cudaFree(s.d_fa);
    s.d_attr = nullptr;
    s.d_fa = nullptr;
    cudaFree(s.gate.ambiguous);  // the bitmaps share its allocation
    cudaFree(s.gate.prob);
    cudaFree(s.gate.feat);
    cudaFree(s.d_front_on);
    cudaFree(s.d_back_on);
    s.gate = GateScratch{};
    s.d_front_on = s.d_back_on = nullptr;
    cudaFree(s.d_s1);
    cudaFree(s.d_resp);
    cudaFree(s.d_counts);
    cudaFree(s.d_cands);
    cudaFree(s.d_ncand);
    cudaFree(s.d_results);
    cudaFree(s.d_win);
    cudaFree(s.D);
    cudaFree(s.R);
    cudaFree(s.M);
    cudaFree(s.F);
    cudaFree(s.first_dec);
    cudaFree(s.survivors);
    cudaFree(s.checked);
    cudaFree(s.d_nraw);
    cudaFree(s.d_faces);
    cudaFree(s.d_nfaces);
    cudaFree(s.d_mk);
    cudaFree(s.d_nmk);
    cudaFreeHost(s.h_nfaces);
    cudaFree(s.d_sync1);
    cudaFreeHost(s.h_faces);
    if (s.done) cudaEventDestroy(s.done);
    if (s.st) cudaStreamDestroy(s.st);
    s = Slot();
}

void Detector::clear() {
    if (!inited_) return;
    cudaSetDevice(device_);
    free_batches();
    for (auto& s : slots_) {
        if (s.st) cudaStreamSynchronize(s.st);
        free_slot(s);
    }
    for (auto& kv : plans_) {
        cudaFree(kv.second->d_levels);
        cudaFree(kv.second->d_chunks);
    }
    plans_.clear();
    scales_.clear();
    inited_ = false;
}

ccnn_status Detector::apply_precision() {
    // paramConverter (CompactCNNLibAPI_v2.cpp:300-326) then Init's precision rules (:922-963)
    type_check_ = 1;
    min_num_detect_ = 1;
    drop_detect_ = api_.drop_detect != 0;
    equalize_ = api_.equalize != 0;
    reflection_ = api_.reflection != 0;
    adapt_min_neighbors_ = false;
    double_check_ = true;
    detect_enabled_ = api_.detect_mode != CCNN_DETECT_DISABLE;
    merger_detect_ = detect_enabled_;
    if (has_cnn_) {
        // CNNDetector's own AdvancedParam instead of the values paramConverter fixes
        type_check_ = cnn_ap_.type_check;
        min_num_detect_ = cnn_ap_.min_num_detect;
        adapt_min_neighbors_ = cnn_ap_.adapt_min_neighbors != 0;
        double_check_ = cnn_ap_.double_check != 0;
        merger_detect_ = cnn_ap_.merger_detect != 0;
    }
    if (api_.detect_precision == CCNN_PRECISION_DEF) {
        gray_image_only_ = true;
        type_check_ = 1;
        equalize_ = true;
        reflection_ = true;
        adapt_min_neighbors_ = true;
        double_check_ = true;
        drop_detect_ = false;
        min_num_detect_ = 1;
        merger_detect_ = true;
    }
    switch (api_.detect_precision) {
        case CCNN_PRECISION_LOW: type_check_ = 0; drop_detect_ = false; break;
        case CCNN_PRECISION_NORMAL: type_check_ = 1; break;
        case CCNN_PRECISION_HIGH: type_check_ = 2; break;
        case CCNN_PRECISION_ULTRA: type_check_ = 2; min_num_detect_ = 2; break;
        default: break;
    }
    if (!detect_enabled_ || api_.facial_analysis) drop_detect_ = false;  // Init (:961-964)
    return CCNN_OK;
}

ccnn_status Detector::create(const ccnn_params& p, const char* const* model_paths, int n_slots, bool colour_input) {
    api_ = p;
    if (n_slots < 1) {
        set_error("a detector needs at least one frame slot");
        return CCNN_ERR_INVALID_ARG;
    }
    slots_.assign(n_slots, Slot());
    for (int i = 0; i < 3; ++i) {
        const char* mp = model_paths ? model_paths[i] : nullptr;
        static const char* kNames[3] = {"cnn4face1_cntk.bin", "cnn4face2_cntk.bin", "cnn4face3_cntk.bin"};
        model_paths_[i] = (mp && mp[0]) ? std::string(mp) : bundled_model_dir() + "/" + kNames[i];
    }
    gray_image_only_ = !colour_input;
    max_w_ = p.max_image_width;
    max_h_ = p.max_image_height;
    return init();
}

ccnn_status Detector::init_host() {
    apply_precision();
    if (max_w_ <= 0 || max_h_ <= 0) {
        set_error("max_image_size must be positive");
        return CCNN_ERR_INVALID_ARG;
    }

    // models (InitCNN / InitCNNCheck). The family follows the files: format 1.0 (`_new.bin`) is
    // the legacy tanh family the reference builds without USE_CNTK_MODELS (then with facial
    // analysis off, cnn_detector_v3.cpp:911-915); otherwise the CNTK format.
    RawModel m[3];
    std::string err;
    {
        std::unique_ptr<LegacyNet[]> lg(new LegacyNet[3]);
        std::string lerr;
        legacy_ = load_legacy_model_file(model_paths_[0], &lg[0], &lerr);
        if (legacy_) {
            for (int i = 1; i < 3; ++i)
                if (!load_legacy_model_file(model_paths_[i], &lg[i], &lerr)) {
                    set_error("legacy cascade: " + lerr + " (all three models must be format 1.0)");
                    return CCNN_ERR_MODEL;
                }
            if (lg[1].min_w != 36 || lg[1].min_h != 40 || lg[2].min_w != 36 || lg[2].min_h != 40) {
                set_error("legacy cascade: stage-2/3 networks must take 36x40 windows");
                return CCNN_ERR_MODEL;
            }
            for (int i = 1; i < 3; ++i)
                if (lg[i].m0 > 6 || lg[i].m2 > 24 || lg[i].hl > 84 || lg[i].k3w != 7 || lg[i].k3h != 8) {
                    set_error("legacy cascade: stage-2/3 networks larger than 6/12/24 maps, 84 hidden neurons or a 7x8 third layer are not supported");
                    return CCNN_ERR_MODEL;
                }
            api_.facial_analysis = 0;
            h_lg_ = std::move(lg);
            for (int i = 0; i < 3; ++i) {
                m[i].min_w = h_lg_[i].min_w;
                m[i].min_h = h_lg_[i].min_h;
            }
        }
    }
    for (int i = 0; i < 3 && !legacy_; ++i)
        if (!load_model_file(model_paths_[i], &m[i], &err)) {
            set_error(err);
            return CCNN_ERR_MODEL;
        }
    if (!wn_) wn_.reset(new WindowNets());
    if (!legacy_ && (!pack_model(m[0], api_.index_output[0], &w1_, &err) || !pack_model(m[1], api_.index_output[1], &wn_->s2, &err) ||
                     !pack_model(m[2], api_.index_output[2], &wn_->s3, &err))) {
        set_error(err);
        return CCNN_ERR_MODEL;
    }
    h_lnet_.reset();
    if (api_.facial_analysis && detect_enabled_) {
        // InitCNNCheck (:792-810): the landmark network, bundled next to the library
        RawModel lm;
        std::unique_ptr<LandmarkNet> ln(new LandmarkNet());
        if (!load_model_file(bundled_model_dir() + "/cnn4landmarks_cntk.bin", &lm, &err) || !pack_landmarks(lm, ln.get(), &err)) {
            set_error(err);
            return CCNN_ERR_MODEL;
        }
        h_lnet_ = std::move(ln);
    }
    pat_w_ = m[0].min_w;
    pat_h_ = m[0].min_h;
    if ((!legacy_ && (pat_w_ != kPatW || pat_h_ != kPatH)) || m[1].min_w != 36 || m[1].min_h != 40 || m[2].min_w != 36 || m[2].min_h != 40) {
        set_error("model window sizes differ from the cascade prototype (23x27 / 36x40)");
        return CCNN_ERR_MODEL;
    }
    if (detect_enabled_) {
        ext_w_ = 36 + kExtOff;
        ext_h_ = 40 + kExtOff;
    } else {
        ext_w_ = pat_w_;
        ext_h_ = pat_h_;
    }

    // InitScales (cnn_detector_v3.cpp:289-346)
    if (!compute_scales(api_, gray_image_only_, pat_h_, max_h_, &scales_, &input_downscale_, &input_scale_)) {
        set_error("invalid configuration: empty scale list");
        return CCNN_ERR_CONFIG;
    }
    if (api_.scale_factor < 1.f) api_.scale_factor = 1.1f;  // InitScales rewrites the parameter (:327-330)
    num_scales_ = (int)scales_.size();

    cfg_.thr1 = api_.treshold[0];
    cfg_.thr2 = api_.treshold[1];
    cfg_.thr3 = api_.treshold[2];
    cfg_.type_check = type_check_;
    cfg_.min_neighbors = api_.min_neighbors;
    cfg_.adapt_min_neighbors = adapt_min_neighbors_;
    cfg_.double_check = double_check_;
    cfg_.drop_detect = drop_detect_;
    cfg_.equalize = equalize_;
    cfg_.reflection = reflection_;
    cfg_.detect_enabled = detect_enabled_;
    cfg_.merger_detect = merger_detect_;
    cfg_.min_num_detect = min_num_detect_;
    cfg_.rescale_output = input_downscale_ ? 1 : 0;
    cfg_.rescale = (float)api_.min_face_height / (float)pat_h_;
    cfg_.pat_w = pat_w_;
    cfg_.pat_h = pat_h_;

    // capacities from the largest plans this configuration can produce
    s1_cap_ = resp_cap_ = img_cap_ = 0;
    k1_cap_ = k2_cap_ = 0;
    chunk_cap_ = 0;
    for (int ch : {1, 3}) {
        Plan tmp;
        ccnn_status st = build_plan(max_w_, max_h_, ch, (int)scales_.size(), &tmp);
        if (st != CCNN_OK) return st;
        s1_cap_ = std::max(s1_cap_, tmp.s1_floats);
        img_cap_ = std::max(img_cap_, tmp.img_floats);
        k1_cap_ = std::max(k1_cap_, tmp.k1_tiles);
        k2_cap_ = std::max(k2_cap_, tmp.k2_tiles);
        resp_cap_ = std::max(resp_cap_, tmp.resp_floats);
        chunk_cap_ = std::max(chunk_cap_, (int)tmp.chunks.size());
    }
    cand_cap_ = std::max(1LL, resp_cap_);
    chunk_cap_ = std::max(chunk_cap_, 1);
    return CCNN_OK;
}

ccnn_status Detector::init() {
    ccnn_status hs = init_host();
    if (hs != CCNN_OK) return hs;
    device_ = api_.cuda_device_id;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        set_error("no CUDA device available (this detector has no CPU path)");
        return CCNN_ERR_CUDA;
    }
    if (device_ < 0 || device_ >= ndev) {
        set_error("cuda_device_id out of range");
        return CCNN_ERR_INVALID_ARG;
    }
    CCNN_CUDA(cudaSetDevice(device_));
    if (legacy_) {
        if (!d_lg_) CCNN_CUDA(cudaMalloc(&d_lg_, 3 * sizeof(LegacyNet)));
        CCNN_CUDA(cudaMemcpy(d_lg_, h_lg_.get(), 3 * sizeof(LegacyNet), cudaMemcpyHostToDevice));
    }
    if (h_lnet_) {
        if (!d_lnet_) CCNN_CUDA(cudaMalloc(&d_lnet_, sizeof(LandmarkNet)));
        CCNN_CUDA(cudaMemcpy(d_lnet_, h_lnet_.get(), sizeof(LandmarkNet), cudaMemcpyHostToDevice));
    }
    if (!order_ev_) CCNN_CUDA(cudaEventCreateWithFlags(&order_ev_, cudaEventDisableTiming));
    cudaDeviceProp prop;
    CCNN_CUDA(cudaGetDeviceProperties(&prop, device_));
    // persistent stage-2/3 grid: 4 resident 256-thread CTAs per SM (register bound)
    window_grid_ = prop.multiProcessorCount * window_ctas_per_sm_;
    facial_grid_ = prop.multiProcessorCount;  // one 118 KB-shared-memory block per SM
    CCNN_CUDA(replay_setup());
    CCNN_CUDA(stage1_setup());
    CCNN_CUDA(window_setup());
    CCNN_CUDA(facial_setup());

    sm_count_ = prop.multiProcessorCount;
    inited_ = true;
    ++init_gen_;
    for (auto& s : slots_) {
        ccnn_status st = alloc_slot(s);
        if (st != CCNN_OK) {
            clear();
            return st;
        }
    }
    ccnn_status bs = alloc_batches();
    if (bs != CCNN_OK) {
        clear();
        return bs;
    }
    return CCNN_OK;
}

ccnn_status Detector::estimate_bytes(const ccnn_params& p, const char* const* model_paths, int n_slots, bool colour_input,
                                     bool with_gate, size_t* bytes) {
    Detector d;
    d.gate_on_ = with_gate;
    d.api_ = p;
    if (n_slots < 1) {
        set_error("a detector needs at least one frame slot");
        return CCNN_ERR_INVALID_ARG;
    }
    d.slots_.assign(n_slots, Slot());
    for (int i = 0; i < 3; ++i) {
        const char* mp = model_paths ? model_paths[i] : nullptr;
        static const char* kNames[3] = {"cnn4face1_cntk.bin", "cnn4face2_cntk.bin", "cnn4face3_cntk.bin"};
        d.model_paths_[i] = (mp && mp[0]) ? std::string(mp) : bundled_model_dir() + "/" + kNames[i];
    }
    d.gray_image_only_ = !colour_input;
    d.max_w_ = p.max_image_width;
    d.max_h_ = p.max_image_height;
    const ccnn_status st = d.init_host();
    if (st != CCNN_OK) return st;
    *bytes = d.slot_bytes();
    return CCNN_OK;
}

// the level arena: only the legacy network reads stored level images (the CNTK stage-1 front kernel
// resamples its tiles from the gray frame)
long long Detector::limg_floats() const { return legacy_ ? std::max(4LL, img_cap_) : 4LL; }

ccnn_status Detector::alloc_slot(Slot& s) {
    CCNN_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
    CCNN_CUDA(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
    s.in_pitch = (size_t)round_up((long long)max_w_ * 4, 64);
    CCNN_CUDA(cudaMalloc(&s.d_in, s.in_pitch * max_h_));
    s.gray_pitch = (int)round_up(max_w_, 16);
    CCNN_CUDA(cudaMalloc(&s.d_gray, sizeof(float) * (size_t)s.gray_pitch * max_h_));
    CCNN_CUDA(cudaMalloc(&s.d_limg, sizeof(float) * limg_floats()));
    CCNN_CUDA(cudaMalloc(&s.d_s1, sizeof(float) * std::max(1LL, s1_cap_)));
    CCNN_CUDA(cudaMalloc(&s.d_resp, sizeof(float) * std::max(1LL, resp_cap_)));
    CCNN_CUDA(cudaMalloc(&s.d_counts, sizeof(int) * chunk_cap_));
    CCNN_CUDA(cudaMalloc(&s.d_cands, sizeof(Candidate) * cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.d_ncand, sizeof(int)));
    CCNN_CUDA(cudaMalloc(&s.d_results, sizeof(CandResult) * cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.d_win, sizeof(WinOut) * 4 * cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.D, sizeof(Det) * cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.R, sizeof(Det) * cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.M, sizeof(Det) * cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.F, sizeof(Det) * cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.first_dec, sizeof(int) * cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.survivors, sizeof(int) * cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.checked, cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.d_nraw, sizeof(int)));
    // at least kHostFaces entries: the per-frame download copies that many
    CCNN_CUDA(cudaMalloc(&s.d_faces, sizeof(FaceOut) * std::max<long long>(cand_cap_, kHostFaces)));
    CCNN_CUDA(cudaMemset(s.d_faces, 0, sizeof(FaceOut) * std::max<long long>(cand_cap_, kHostFaces)));
    CCNN_CUDA(cudaMalloc(&s.d_nfaces, sizeof(int)));
    CCNN_CUDA(cudaMalloc(&s.d_mk, sizeof(Det) * cand_cap_));
    CCNN_CUDA(cudaMalloc(&s.d_nmk, sizeof(int)));
    if (gate_on_) {
        ccnn_status st = alloc_gate(s);
        if (st != CCNN_OK) return st;
    }
    if (d_lnet_ && api_.facial_analysis) {
        CCNN_CUDA(cudaMalloc(&s.d_attr, sizeof(int4) * cand_cap_));
        CCNN_CUDA(cudaMalloc(&s.d_fa, sizeof(int) * 5 * cand_cap_));
    }
    CCNN_CUDA(cudaMallocHost(&s.h_nfaces, 2 * sizeof(int)));
    s.h_nfaces[1] = 0;
    CCNN_CUDA(cudaMalloc(&s.d_sync1, sizeof(int) * (2 + kBatchStages)));
    CCNN_CUDA(cudaMallocHost(&s.h_faces, sizeof(FaceOut) * kHostFaces));
    CCNN_CUDA(cudaMemsetAsync(s.d_ncand, 0, sizeof(int), s.st));
    CCNN_CUDA(cudaMemsetAsync(s.d_nraw, 0, sizeof(int), s.st));
    CCNN_CUDA(cudaMemsetAsync(s.d_nfaces, 0, sizeof(int), s.st));
    return CCNN_OK;
}

ccnn_status Detector::build_plan(int w, int h, int ch, int num_scales, Plan* p) {
    p->in_w = w;
    p->in_h = h;
    p->ch = ch;
    p->in_pitch = (size_t)round_up((long long)w * ch, 64);
    p->downscale = input_downscale_ && ch == 1;
    if (p->downscale)
        size_scale(w, h, input_scale_, &p->gw, &p->gh);
    else {
        p->gw = w;
        p->gh = h;
    }
    p->levels.clear();
    p->chunks.clear();
    long long s1 = 0, resp = 0, img = 0;
    int k1 = 0, k2 = 0, pyr = 0;
    int n = 0;
    for (int scl = 0; scl < num_scales && scl < (int)scales_.size(); ++scl) {
        LevelDesc L{};
        size_scale(p->gw, p->gh, scales_[scl], &L.w, &L.h);
        if (L.w < ext_w_ || L.h < ext_h_) break;  // this and every smaller level are skipped
        L.mode = (L.w == p->gw && L.h == p->gh) ? 0 : (scales_[scl] > 0.7f ? 1 : 2);
        L.sclx = ((uint32_t)p->gw << 12) / (uint32_t)L.w + 1u;
        L.scly = ((uint32_t)p->gh << 12) / (uint32_t)L.h + 1u;
        L.scale = scales_[scl];
        L.inv_scale = 1.f / scales_[scl];
        L.p1w = (L.w - 3) >> 1;
        L.p1h = (L.h - 3) >> 1;
        L.p2w = (L.p1w - 2) >> 1;
        L.p2h = (L.p1h - 2) >> 1;
        L.ow = L.p2w - 3;
        L.oh = L.p2h - 4;
        L.s1_pitch = (int)round_up(L.p1w, 32);
        L.s1_plane = (long long)L.s1_pitch * L.p1h;
        L.s1_off = s1;
        s1 += 4 * L.s1_plane;
        if (legacy_) {
            // the legacy stage-1 network's response map, and its pooled L1 and L2 maps in the S1 arena
            const LegacyNet& n = h_lg_[0];
            legacy_output_size(n, L.w, L.h, &L.ow, &L.oh);
            s1 -= 4 * L.s1_plane;  // L.s1_off stays this level's start
            s1 += (long long)n.m0 * L.p1w * L.p1h + (long long)n.m1 * L.p2w * L.p2h;
        }
        L.resp_off = resp;
        resp += (long long)L.ow * L.oh;
        L.k1_tiles_x = (L.p1w + kK1TileX - 1) / kK1TileX;
        L.k1_base = k1;
        k1 += L.k1_tiles_x * ((L.p1h + kK1TileY - 1) / kK1TileY);
        L.k2_tiles_x = (L.ow + kK2TileX - 1) / kK2TileX;
        L.k2_base = k2;
        k2 += L.k2_tiles_x * ((L.oh + kK2TileY - 1) / kK2TileY);
        L.img_pitch = (int)round_up(L.w, 4);
        L.img_vec = 1;
        L.img_off = img;
        img += (long long)L.img_pitch * L.h;
        L.pyr_wq = (L.img_pitch + kPyrCols - 1) / kPyrCols;
        L.pyr_base = pyr;
        pyr += L.pyr_wq * ((L.h + kPyrRows - 1) / kPyrRows);
        p->levels.push_back(L);
        ++n;
    }
    p->n_levels = n;
    for (int scl = n - 1; scl >= 0; --scl) {
        LevelDesc& L = p->levels[scl];
        L.order = n - 1 - scl;
        L.chunk_base = (int)p->chunks.size();
        L.octave = (int)std::floor(std::log2((double)scales_[0] / (double)scales_[scl]) + 1e-9);
        const int total = L.ow * L.oh;
        for (int s = 0; s < total; s += kCandChunk) p->chunks.push_back(make_int4(scl, s, std::min(kCandChunk, total - s), 0));
    }
    p->k1_tiles = k1;
    p->k2_tiles = k2;
    p->s1_floats = s1;
    p->resp_floats = resp;
    p->img_floats = img;
    return CCNN_OK;
}

// Resolves the pyramid plan of a frame and advances num_scales as RunCPUDetect does.
ccnn_status Detector::plan_for(int w, int h, int ch, const Plan** out) {
    const bool downscale = input_downscale_ && ch == 1;
    auto key = std::make_tuple(w, h, downscale ? 1 : 3, num_scales_);
    auto it = plans_.find(key);
    if (it == plans_.end()) {
        std::unique_ptr<Plan> p(new Plan());
        ccnn_status st = build_plan(w, h, ch, num_scales_, p.get());
        if (st != CCNN_OK) return st;
        if (p->s1_floats > s1_cap_ || p->resp_floats > resp_cap_ || p->img_floats > img_cap_ ||
            (long long)p->chunks.size() > chunk_cap_) {
            set_error("internal: pyramid plan exceeds the allocated buffers");
            return CCNN_ERR_CUDA;
        }
        if (p->n_levels > 0) {
            CCNN_CUDA(cudaMalloc(&p->d_levels, sizeof(LevelDesc) * p->n_levels));
            CCNN_CUDA(cudaMemcpy(p->d_levels, p->levels.data(), sizeof(LevelDesc) * p->n_levels, cudaMemcpyHostToDevice));
        }
        if (!p->chunks.empty()) {
            CCNN_CUDA(cudaMalloc(&p->d_chunks, sizeof(int4) * p->chunks.size()));
            CCNN_CUDA(cudaMemcpy(p->d_chunks, p->chunks.data(), sizeof(int4) * p->chunks.size(), cudaMemcpyHostToDevice));
        }
        it = plans_.emplace(key, std::move(p)).first;
    }
    const Plan* p = it->second.get();
    // a level too small for the stage-2/3 window lowers num_scales for later frames (:2086)
    if (p->n_levels < num_scales_) num_scales_ = p->n_levels;
    *out = p;
    return CCNN_OK;
}

ccnn_status Detector::alloc_gate(Slot& s) {
    if (s.gate.prob) return CCNN_OK;
    const size_t w8 = (size_t)max_w_ / 8, h8 = (size_t)max_h_ / 8;
    const size_t cells = (w8 / 2) * (h8 / 2);
    void* words = nullptr;
    CCNN_CUDA(cudaMalloc(&words, sizeof(uint32_t) * (1 + (size_t)gate_bitmap_words(max_w_, max_h_))));
    s.gate.ambiguous = (int*)words;
    s.gate.bits = (uint32_t*)words + 1;
    CCNN_CUDA(cudaMalloc(&s.gate.prob, sizeof(float) * std::max<size_t>(1, kGK * cells)));
    CCNN_CUDA(cudaMalloc(&s.gate.feat, sizeof(__half) * std::max<size_t>(1, w8 * h8)));
    CCNN_CUDA(cudaMalloc(&s.d_front_on, std::max(1, k1_cap_)));
    CCNN_CUDA(cudaMalloc(&s.d_back_on, std::max(1, k2_cap_)));
    return CCNN_OK;
}

ccnn_status Detector::gate_set(const float* params, int n, float threshold, float fallback_fraction) {
    std::lock_guard<std::mutex> lk(mu_);
    if (!params || n != kGateParams || !(threshold > 0.f && threshold < 1.f) || !(fallback_fraction >= 0.f)) {
        set_error("gate: kGateParams parameters, a threshold in (0, 1) and a non-negative fallback fraction are needed");
        return CCNN_ERR_INVALID_ARG;
    }
    if (!inited_) {
        ccnn_status st = init();
        if (st != CCNN_OK) return st;
    }
    if (legacy_) {
        set_error("gate: the learned gate is trained for the CNTK cascade, not the legacy model family");
        return CCNN_ERR_UNSUPPORTED;
    }
    cudaSetDevice(device_);
    gate_params_.assign(params, params + n);
    std::copy(params, params + kGateParams, gate_net_.p);
    gate_on_ = true;
    gate_thr_ = threshold;
    gate_amb_frac_ = fallback_fraction;
    for (auto& s : slots_) {
        if (s.st) CCNN_CUDA(cudaStreamSynchronize(s.st));
        ccnn_status st = alloc_gate(s);
        if (st != CCNN_OK) return st;
        s.exec_plan = nullptr;  // the per-frame graphs are captured again with the gate
    }
    for (auto& b : batches_) b.exec_plan = nullptr;  // and the batched ones (their streams are the slots')
    return CCNN_OK;
}

ccnn_status Detector::set_schedule(int frame_slots, int window_ctas_per_sm, int front_bpsm, int back_bpsm, int batch_frames, int batch_bpsm) {
    std::lock_guard<std::mutex> lk(mu_);
    const int slots = frame_slots > 0 ? frame_slots : (int)slots_.size();
    const int batch = batch_frames >= 0 ? batch_frames : batch_frames_;
    if (frame_slots < 0 || frame_slots > 64 || window_ctas_per_sm < 0 || window_ctas_per_sm > 6 || (front_bpsm != 0 && (front_bpsm < 3 || front_bpsm > 4)) ||
        (back_bpsm != 0 && (back_bpsm < 3 || back_bpsm > 4)) || (batch_bpsm != 0 && (batch_bpsm < 1 || batch_bpsm > 4)) || batch > kMaxBatch ||
        (batch > 1 && slots < batch)) {
        set_error("schedule: 1-64 frame slots, 1-6 stage-2/3 blocks per SM, 3-4 stage-1 blocks per SM, batches of 0-16 frames, "
                  "1-4 persistent stage-1 blocks per SM and at least as many frame slots as frames per batch (0 keeps the "
                  "current value)");
        return CCNN_ERR_INVALID_ARG;
    }
    clear();
    if (frame_slots > 0) slots_.assign(frame_slots, Slot());
    if (window_ctas_per_sm > 0) window_ctas_per_sm_ = window_ctas_per_sm;
    if (front_bpsm > 0) s1_sched_.front_blocks_per_sm = front_bpsm;
    if (back_bpsm > 0) s1_sched_.back_blocks_per_sm = back_bpsm;
    if (batch_frames >= 0) batch_frames_ = batch_frames;
    if (batch_bpsm > 0) batch_bpsm_ = batch_bpsm;
    return init();
}

void Detector::get_schedule(int* frame_slots, int* window_ctas_per_sm, int* front_bpsm, int* back_bpsm, int* batch_frames, int* batch_bpsm) const {
    *frame_slots = (int)slots_.size();
    *window_ctas_per_sm = window_ctas_per_sm_;
    if (front_bpsm) *front_bpsm = s1_sched_.front_blocks_per_sm;
    if (back_bpsm) *back_bpsm = s1_sched_.back_blocks_per_sm;
    if (batch_frames) *batch_frames = batch_frames_;
    if (batch_bpsm) *batch_bpsm = batch_bpsm_;
}

ccnn_status Detector::gate_set_margin(int pixels) {
    std::lock_guard<std::mutex> lk(mu_);
    if (pixels < 0 || pixels > 64) {
        set_error("gate margin: 0-64 pixels");
        return CCNN_ERR_INVALID_ARG;
    }
    gate_margin_ = pixels;
    for (auto& s : slots_) {
        if (s.st) cudaStreamSynchronize(s.st);
        s.exec_plan = nullptr;  // the per-frame graphs are captured again with the new margin
    }
    for (auto& b : batches_) b.exec_plan = nullptr;
    return CCNN_OK;
}

ccnn_status Detector::gate_disable() {
    std::lock_guard<std::mutex> lk(mu_);
    gate_on_ = false;
    for (auto& s : slots_) {
        if (s.st) cudaStreamSynchronize(s.st);
        s.exec_plan = nullptr;
    }
    for (auto& b : batches_) b.exec_plan = nullptr;
    return CCNN_OK;
}

ccnn_status Detector::gate_labels(uint8_t* d_labels, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(mu_);
    Slot& s = slots_[0];
    if (!inited_ || !s.last_plan || !detect_enabled_) {
        set_error("no frame has been processed with stages 2 and 3");
        return CCNN_ERR_INVALID_ARG;
    }
    cudaSetDevice(device_);
    CCNN_CUDA(cudaStreamSynchronize(s.st));
    const Plan& p = *s.last_plan;
    CCNN_CUDA(launch_gate_labels(s.d_cands, s.d_results, s.d_ncand, (int)cand_cap_, p.d_levels, p.gw, p.gh, d_labels, st));
    return CCNN_OK;
}

ccnn_status Detector::gate_stats(int* front_run, int* front_total, int* back_run, int* back_total, int* fallback) {
    std::lock_guard<std::mutex> lk(mu_);
    Slot& s = slots_[0];
    if (!inited_ || !s.last_plan) {
        set_error("no frame has been processed");
        return CCNN_ERR_INVALID_ARG;
    }
    cudaSetDevice(device_);
    CCNN_CUDA(cudaStreamSynchronize(s.st));
    const Plan& p = *s.last_plan;
    *fallback = 0;
    if (p.n_levels <= 0) {  // a frame too small for any level scans nothing
        *front_run = *front_total = *back_run = *back_total = 0;
        return CCNN_OK;
    }
    const LevelDesc& last = p.levels[p.n_levels - 1];
    const int nb = last.k2_base + last.k2_tiles_x * ((last.oh + kK2TileY - 1) / kK2TileY);
    const int nf = last.k1_base + last.k1_tiles_x * ((last.p1h + kK1TileY - 1) / kK1TileY);
    *front_total = nf;
    *back_total = nb;
    *front_run = nf;
    *back_run = nb;
    *fallback = 0;
    if (!gate_on_ || !s.gate.prob || p.gw < 32 || p.gh < 32) return CCNN_OK;
    std::vector<uint8_t> f(nf), b(nb);
    CCNN_CUDA(cudaMemcpy(f.data(), s.d_front_on, nf, cudaMemcpyDeviceToHost));
    CCNN_CUDA(cudaMemcpy(b.data(), s.d_back_on, nb, cudaMemcpyDeviceToHost));
    int amb = 0;
    CCNN_CUDA(cudaMemcpy(&amb, s.gate.ambiguous, sizeof(int), cudaMemcpyDeviceToHost));
    *front_run = (int)std::count(f.begin(), f.end(), (uint8_t)1);
    *back_run = (int)std::count(b.begin(), b.end(), (uint8_t)1);
    const int w16 = (p.gw / 8) / 2, h16 = (p.gh / 8) / 2;
    *fallback = amb > (int)(gate_amb_frac_ * (float)(w16 * h16 * kGK)) ? 1 : 0;
    return CCNN_OK;
}

ccnn_status Detector::gate_probabilities(float* out, int cap, int* n) {
    std::lock_guard<std::mutex> lk(mu_);
    Slot& s = slots_[0];
    if (!inited_ || !s.last_plan) {
        set_error("no frame has been processed");
        return CCNN_ERR_INVALID_ARG;
    }
    const Plan& p = *s.last_plan;
    if (!gate_on_ || !s.gate.prob || p.gw < 32 || p.gh < 32) {
        set_error("the last frame ran without the learned gate");
        return CCNN_ERR_INVALID_ARG;
    }
    cudaSetDevice(device_);
    CCNN_CUDA(cudaStreamSynchronize(s.st));
    const int total = kGK * ((p.gw / 8) / 2) * ((p.gh / 8) / 2);
    *n = total;
    if (out && cap > 0) CCNN_CUDA(cudaMemcpy(out, s.gate.prob, sizeof(float) * std::min(cap, total), cudaMemcpyDeviceToHost));
    return cap < total ? CCNN_TRUNCATED : CCNN_OK;
}

ReplayArgs Detector::replay_args(Slot& s, const Plan& p) const {
    ReplayArgs a;
    a.cands = s.d_cands;
    a.n_cand = s.d_ncand;
    a.win = s.d_win;
    a.results = s.d_results;
    a.levels = p.d_levels;
    a.n_levels = p.n_levels;
    a.cfg = cfg_;
    a.D = s.D;
    a.R = s.R;
    a.M = s.M;
    a.F = s.F;
    a.first_dec = s.first_dec;
    a.survivors = s.survivors;
    a.checked = s.checked;
    a.attr = s.d_attr;
    a.fa_scratch = s.d_fa;
    a.n_raw = s.d_nraw;
    a.faces = s.d_faces;
    a.face_cap = (int)cand_cap_;
    a.n_faces = s.d_nfaces;
    a.m_out = s.d_mk;
    a.n_m_out = s.d_nmk;
    return a;
}

ccnn_status Detector::enqueue_kernels(Slot& s, const Plan& p) {
    // the learned gate decides which stage-1 tiles run, and so which parts of the pyramid are read;
    // the gray launch also writes its input features
    const bool gated = gate_on_ && s.gate.prob && p.gw >= 32 && p.gh >= 32;
    s.gray_feat = (gated && !p.downscale) ? s.gate.feat : nullptr;
    cudaError_t e;
    if (p.downscale)
        e = launch_gray_u8_resized(s.d_in, (int)p.in_pitch, p.in_w, p.in_h, s.d_gray, s.gray_pitch, p.gw, p.gh, s.st);
    else
        e = launch_gray(s.d_in, (int)p.in_pitch, p.in_w, p.in_h, p.ch, s.d_gray, s.gray_pitch, s.st, s.gray_feat);
    CCNN_CUDA(e);
    if (gated) {
        CCNN_CUDA(launch_gate(gate_net_, s.d_gray, s.gray_pitch, p.gw, p.gh, s.gray_feat != nullptr, p.levels.data(), p.n_levels, s.gate,
                              gate_thr_, gate_amb_frac_, gate_margin_, s.d_back_on, s.d_front_on, s.st));
    }
    const bool single = single_launch_stage1() && p.n_levels > 0 && p.n_levels <= kMaxBatchLevels;
    if (single) {
        // the pyramid and stage 1 of every level in one persistent launch (the batched form's kernel on
        // one frame; front tiles resample their level tiles from the gray frame): what the reference's
        // level atlas (packet mode) is for
        BatchFrames F{};
        F.gray[0] = s.d_gray;
        F.gpitch = s.gray_pitch;
        F.gw = p.gw;
        F.gh = p.gh;
        F.s1[0] = s.d_s1;
        F.resp[0] = s.d_resp;
        F.counts[0] = s.d_counts;
        F.front_on[0] = gated ? s.d_front_on : nullptr;
        F.back_on[0] = gated ? s.d_back_on : nullptr;
        F.cells[0] = gated ? gate_cells(s.gate, p.gw, p.gh, gate_amb_frac_, gate_margin_) : GateCells{};
        if (!p.chunks.empty()) CCNN_CUDA(cudaMemsetAsync(s.d_counts, 0, sizeof(int) * p.chunks.size(), s.st));
        BatchQueue Q;
        build_batch_queue(&Q, 1, p.n_levels, (int)p.chunks.size(), p.k1_tiles, p.k2_tiles, cfg_.thr1);
        CCNN_CUDA(cudaMemsetAsync(s.d_sync1, 0, sizeof(int) * (2 + kBatchStages), s.st));
        CCNN_CUDA(launch_stage1_batch(w1_, F, Q, p.d_levels, s.d_sync1, s.d_sync1 + 1 + kBatchStages,
                                      sm_count_ * stage1_batch_blocks_per_sm(batch_bpsm_), s.st, batch_bpsm_));
        CCNN_CUDA(cudaMemcpyAsync(s.h_nfaces + 1, s.d_sync1 + 1 + kBatchStages, sizeof(int), cudaMemcpyDeviceToHost, s.st));
    } else {
        // the legacy network reads stored level images; the CNTK front kernel resamples its tiles from
        // the gray frame itself
        if (legacy_) CCNN_CUDA(launch_pyramid(p.levels.data(), p.n_levels, s.d_gray, s.gray_pitch, p.gw, p.gh, s.d_limg, s.st));
        // the back kernel counts each chunk's candidates as it writes the responses
        if (!p.chunks.empty()) CCNN_CUDA(cudaMemsetAsync(s.d_counts, 0, sizeof(int) * p.chunks.size(), s.st));
    }
    if (!single) {
        if (legacy_) {
            const ccnn_status ls = enqueue_legacy_stage1(s, p);
            if (ls != CCNN_OK) return ls;
        } else {
            CCNN_CUDA(launch_stage1(w1_, p.levels.data(), p.n_levels, nullptr, s.d_s1, s.d_resp, s.st, s.d_counts, cfg_.thr1,
                                    gated ? s.d_front_on : nullptr, gated ? s.d_back_on : nullptr,
                                    gated ? gate_cells(s.gate, p.gw, p.gh, gate_amb_frac_, gate_margin_) : GateCells{}, s1_sched_,
                                    GrayRef{s.d_gray, s.gray_pitch, p.gw, p.gh}));
        }
    }
    CCNN_CUDA(launch_cand_write(p.d_chunks, (int)p.chunks.size(), p.d_levels, s.d_resp, cfg_.thr1, s.d_counts, s.d_cands, s.d_ncand,
                                (int)cand_cap_, s.st));
    if (detect_enabled_)
        CCNN_CUDA(launch_window(*wn_, s.d_gray, s.gray_pitch, p.gw, p.gh, s.d_cands, s.d_ncand, p.d_levels, s.d_win, cfg_,
                                window_grid_, s.st, legacy_ ? d_lg_ : nullptr, window_ctas_per_sm_));
    if (s.d_attr)
        CCNN_CUDA(launch_facial(d_lnet_, s.d_gray, s.gray_pitch, p.gw, p.gh, s.d_cands, s.d_ncand, p.d_levels, s.d_win, cfg_, s.d_attr,
                                facial_grid_, s.st));
    CCNN_CUDA(launch_replay(replay_args(s, p), s.st));
    CCNN_CUDA(cudaMemcpyAsync(s.h_nfaces, s.d_nfaces, sizeof(int), cudaMemcpyDeviceToHost, s.st));
    CCNN_CUDA(cudaMemcpyAsync(s.h_faces, s.d_faces, sizeof(FaceOut) * kGraphFaces, cudaMemcpyDeviceToHost, s.st));
    return CCNN_OK;
}

// Stage 1 of the legacy family: the legacy network on every level image, its pooled maps in the
// S1 arena, candidates counted per scan chunk.
ccnn_status Detector::enqueue_legacy_stage1(Slot& s, const Plan& p) {
    for (int i = 0; i < p.n_levels; ++i) {
        const LevelDesc& L = p.levels[i];
        CCNN_CUDA(launch_legacy_forward(d_lg_, h_lg_[0], s.d_limg + L.img_off, L.img_pitch, L.w, L.h, s.d_s1 + L.s1_off, s.d_resp + L.resp_off, s.st,
                                        s.d_counts, L.chunk_base, cfg_.thr1));
    }
    return CCNN_OK;
}

// Points the graph's gray-conversion node at `src` (row pitch `spitch` bytes) for the next launches.
static cudaError_t retarget_gray(Slot& s, const Plan& p, const uint8_t* src, int spitch) {
    int w = p.in_w, h = p.in_h, dpitch = s.gray_pitch;
    float* dst = s.d_gray;
    __half* feat = s.gray_feat;
    void* args[7] = {&src, &spitch, &w, &h, &dst, &dpitch, &feat};
    cudaKernelNodeParams kp = s.gray_kp;
    kp.kernelParams = args;
    kp.extra = nullptr;
    return cudaGraphExecKernelNodeSetParams(s.exec, s.gray_node, &kp);
}

ccnn_status Detector::enqueue(Slot& s, const Plan& p, const ccnn_image& img, bool device_input, cudaStream_t) {
    if (s.exec_plan != &p) {
        if (s.exec) {
            cudaGraphExecDestroy(s.exec);
            s.exec = nullptr;
        }
        if (s.graph) {
            cudaGraphDestroy(s.graph);
            s.graph = nullptr;
        }
        s.gray_node = nullptr;
        s.gray_in_place = false;
        cudaGraph_t g;
        CCNN_CUDA(cudaStreamBeginCapture(s.st, cudaStreamCaptureModeThreadLocal));
        ccnn_status st = enqueue_kernels(s, p);
        cudaError_t ce = cudaStreamEndCapture(s.st, &g);
        if (st != CCNN_OK) return st;
        CCNN_CUDA(ce);
        ce = cudaGraphInstantiate(&s.exec, g, 0);
        if (ce != cudaSuccess) cudaGraphDestroy(g);
        CCNN_CUDA(ce);
        s.graph = g;
        s.exec_plan = &p;
        // the gray-conversion node, so that device frames can be read where they are
        if (!p.downscale) {
            size_t nn = 0;
            CCNN_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
            std::vector<cudaGraphNode_t> nodes(nn);
            if (nn) CCNN_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
            const void* fn = gray_kernel_fn(p.ch, s.gray_feat != nullptr);
            for (cudaGraphNode_t nd : nodes) {
                cudaGraphNodeType t;
                CCNN_CUDA(cudaGraphNodeGetType(nd, &t));
                if (t != cudaGraphNodeTypeKernel) continue;
                cudaKernelNodeParams kp;
                CCNN_CUDA(cudaGraphKernelNodeGetParams(nd, &kp));
                if (kp.func == fn) {
                    s.gray_node = nd;
                    s.gray_kp = kp;
                    break;
                }
            }
        }
    }
    // A device frame with the gray kernel's alignment (64-byte base and step) is read in place;
    // anything else is packed into the slot's input buffer at the plan's pitch, as one contiguous
    // copy when the frame's step already is that pitch (the copy engines move it faster than rows).
    const bool in_place = device_input && s.gray_node && !((uintptr_t)img.data & 63) && !(img.step & 63) && img.step <= (size_t)INT32_MAX;
    if (in_place) {
        CCNN_CUDA(retarget_gray(s, p, (const uint8_t*)img.data, (int)img.step));
        s.gray_in_place = true;
    } else {
        if (s.gray_in_place) {
            CCNN_CUDA(retarget_gray(s, p, s.d_in, (int)p.in_pitch));
            s.gray_in_place = false;
        }
        const size_t row = (size_t)img.cols * img.channels;
        const cudaMemcpyKind kind = device_input ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        if (img.step == p.in_pitch)
            CCNN_CUDA(cudaMemcpyAsync(s.d_in, img.data, p.in_pitch * (size_t)(img.rows - 1) + row, kind, s.st));
        else
            CCNN_CUDA(cudaMemcpy2DAsync(s.d_in, p.in_pitch, img.data, img.step, row, img.rows, kind, s.st));
    }
    s.last_in_place = in_place;
    CCNN_CUDA(cudaGraphLaunch(s.exec, s.st));
    CCNN_CUDA(cudaEventRecord(s.done, s.st));
    s.last_plan = &p;
    return CCNN_OK;
}

// Waits for slot s's frame and returns its faces: the graph downloads the first kGraphFaces; more
// (up to `cap`) are fetched here. *src points at `cap`-or-fewer FaceOut entries valid until the
// next call on the slot.
ccnn_status Detector::collect_raw(Slot& s, int cap, int* n, const FaceOut** src) {
    CCNN_CUDA(cudaEventSynchronize(s.done));
    CCNN_CUDA(cudaGetLastError());
    if (s.h_nfaces[1] != 0) {
        s.h_nfaces[1] = 0;
        set_error("single-launch stage 1: a dependency wait gave up (the frame's results are invalid)");
        return CCNN_ERR_CUDA;
    }
    const int nf = *s.h_nfaces;
    *n = nf;
    const int take = std::min(nf, cap);
    *src = s.h_faces;
    if (take > kGraphFaces) {
        if (take > kHostFaces) {
            s.h_extra.resize(take);
            CCNN_CUDA(cudaMemcpy(s.h_extra.data(), s.d_faces, sizeof(FaceOut) * take, cudaMemcpyDeviceToHost));
            *src = s.h_extra.data();
        } else {
            CCNN_CUDA(cudaMemcpy(s.h_faces + kGraphFaces, s.d_faces + kGraphFaces, sizeof(FaceOut) * (take - kGraphFaces),
                                 cudaMemcpyDeviceToHost));
        }
    }
    return CCNN_OK;
}

ccnn_status Detector::collect(Slot& s, ccnn_face* faces, int cap, int* n) {
    const FaceOut* src = nullptr;
    ccnn_status st = collect_raw(s, cap, n, &src);
    if (st != CCNN_OK) return st;
    const int nf = *n;
    const int take = std::min(nf, cap);
    for (int i = 0; i < take; ++i) {
        faces[i].x = src[i].x;
        faces[i].y = src[i].y;
        faces[i].width = src[i].w;
        faces[i].height = src[i].h;
        faces[i].score = src[i].score;
        faces[i].gender = src[i].gender;
        faces[i].smile = src[i].smile;
        faces[i].glasses = src[i].glasses;
    }
    return nf > cap ? CCNN_TRUNCATED : CCNN_OK;
}

// Frame admission: the reference's size and channel rules, then the frame's plan.
ccnn_status Detector::prepare_frame(const ccnn_image& img, const Plan** plan, bool* empty) {
    *empty = false;
    if (img.cols <= 0 || img.rows <= 0 || !img.data || img.step < (size_t)img.cols * img.channels) {
        set_error("invalid image");
        return CCNN_ERR_INVALID_ARG;
    }
    if (img.channels != 1 && img.channels != 3 && img.channels != 4) {
        set_error("this type of image is not supported (1, 3 or 4 channels)");
        return CCNN_ERR_UNSUPPORTED;
    }
    if (!inited_) {
        ccnn_status st = init();
        if (st != CCNN_OK) return st;
    }
    if (img.cols < ext_w_ || img.rows < ext_h_) {
        *empty = true;
        return CCNN_OK;
    }
    if (img.cols > max_w_ || img.rows > max_h_) {
        clear();
        max_w_ = img.cols;
        max_h_ = img.rows;
        if (gray_image_only_ && img.channels != 1) gray_image_only_ = false;
        ccnn_status st = init();
        if (st != CCNN_OK) return st;
    } else if (img.cols != max_w_ || img.rows != max_h_) {
        num_scales_ = (int)scales_.size();
    }
    if (gray_image_only_ && input_downscale_ && img.channels != 1) {
        gray_image_only_ = false;
        clear();
        ccnn_status st = init();
        if (st != CCNN_OK) return st;
        if (gray_image_only_ && input_downscale_) {
            // precision `def` forces gray_image_only back on in Init; the reference then recurses
            // without end (cnn_detector_v3.cpp:2540-2545 with :924-926)
            set_error("precision 'def' with a colour frame needs min_face_height < 34 (the reference recurses forever)");
            return CCNN_ERR_CONFIG;
        }
    }
    return plan_for(img.cols, img.rows, img.channels, plan);
}

ccnn_status Detector::detect(const ccnn_image& img, bool device_input, cudaStream_t user_stream, ccnn_face* faces, int cap, int* n) {
    std::lock_guard<std::mutex> lk(mu_);
    if (!n || (cap > 0 && !faces) || cap < 0) {
        set_error("invalid output arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    cudaSetDevice(device_);
    const Plan* p = nullptr;
    bool empty = false;
    ccnn_status st = prepare_frame(img, &p, &empty);
    if (st != CCNN_OK) return st;
    if (empty) {
        *n = 0;
        return CCNN_OK;
    }
    Slot& s = slots_[0];
    // a device frame is read on the slot's stream: order it after the caller's pending work on its
    // stream (the legacy default stream when none is given), which may still be writing the frame
    if (device_input) {
        st = order_after(user_stream, 1);
        if (st != CCNN_OK) return st;
    }
    st = enqueue(s, *p, img, device_input, user_stream);
    if (st != CCNN_OK) return st;
    return collect(s, faces, cap, n);
}

ccnn_status Detector::order_after(cudaStream_t user_stream, int n_slots) {
    CCNN_CUDA(cudaEventRecord(order_ev_, user_stream ? user_stream : cudaStreamLegacy));
    for (int k = 0; k < n_slots && k < (int)slots_.size(); ++k) CCNN_CUDA(cudaStreamWaitEvent(slots_[k].st, order_ev_, 0));
    return CCNN_OK;
}

ccnn_status Detector::launch(int k, const ccnn_image& img) {
    if (k < 0 || k >= (int)slots_.size()) {
        set_error("slot index out of range");
        return CCNN_ERR_INVALID_ARG;
    }
    if (img.cols != max_w_ || img.rows != max_h_ || (gray_image_only_ && img.channels != 1)) {
        set_error("frame does not match the slot configuration");
        return CCNN_ERR_INVALID_ARG;
    }
    cudaSetDevice(device_);
    const Plan* p = nullptr;
    bool empty = false;
    ccnn_status st = prepare_frame(img, &p, &empty);
    if (st != CCNN_OK) return st;
    if (empty) {  // no level fits the stage-2/3 window: an empty result, nothing launched
        *slots_[k].h_nfaces = 0;
        CCNN_CUDA(cudaEventRecord(slots_[k].done, slots_[k].st));
        return CCNN_OK;
    }
    return enqueue(slots_[k], *p, img, false, nullptr);
}

bool Detector::slot_done(int k) { return cudaEventQuery(slots_[k].done) != cudaErrorNotReady; }

ccnn_status Detector::fetch(int k, ccnn_face* faces, int cap, int* n) { return collect(slots_[k], faces, cap, n); }

size_t Detector::slot_bytes() const {
    const size_t in = (size_t)round_up((long long)max_w_ * 4, 64) * max_h_;
    const size_t gray = sizeof(float) * (size_t)round_up(max_w_, 16) * max_h_;
    const size_t per_cand = sizeof(Candidate) + sizeof(CandResult) + 4 * sizeof(WinOut) + 5 * sizeof(Det) + 2 * sizeof(int) + 1;
    size_t per_slot = in + gray + sizeof(float) * (size_t)(limg_floats() + std::max(1LL, s1_cap_) + std::max(1LL, resp_cap_)) +
                      sizeof(int) * chunk_cap_ + per_cand * (size_t)cand_cap_ + sizeof(FaceOut) * std::max<long long>(cand_cap_, kHostFaces);
    if (gate_on_) {
        const size_t cells = ((size_t)max_w_ / 16) * ((size_t)max_h_ / 16);
        per_slot += sizeof(uint32_t) * (1 + (size_t)gate_bitmap_words(max_w_, max_h_)) + sizeof(float) * std::max<size_t>(1, kGK * cells) +
                    sizeof(__half) * std::max<size_t>(1, ((size_t)max_w_ / 8) * ((size_t)max_h_ / 8)) +
                    (size_t)std::max(1, k1_cap_) + (size_t)std::max(1, k2_cap_);
    }
    if (h_lnet_) per_slot += (sizeof(int4) + 5 * sizeof(int)) * (size_t)cand_cap_;
    return per_slot * slots_.size();
}

ccnn_status Detector::detect_batch(const ccnn_image* imgs, int n_img, bool device_input, ccnn_face* faces, int cap_per, int* n_faces,
                                   float* gpu_ms) {
    std::lock_guard<std::mutex> lk(mu_);
    if (n_img < 0 || (n_img > 0 && (!imgs || !n_faces)) || cap_per < 0 || (cap_per > 0 && n_img > 0 && !faces)) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    cudaSetDevice(device_);
    const int n_sl = (int)slots_.size();
    std::vector<int> pending(n_sl, -1);
    // device frames: a slot stream waits for the work queued on the legacy default stream (where a
    // caller without a stream of its own, torch included, wrote them) before its first frame of the
    // batch, and again after a re-initialisation recreated the slots
    int ordered_gen = -1;
    std::vector<char> waited(n_sl, 0);
    ccnn_status worst = CCNN_OK;
    // device time of the whole batch: from an event before the first frame's upload (both
    // slot streams wait on it) to an event after the last frame of either slot
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (gpu_ms && inited_) {
        CCNN_CUDA(cudaEventCreate(&t0));
        CCNN_CUDA(cudaEventCreate(&t1));
        CCNN_CUDA(cudaEventRecord(t0, slots_[0].st));
        for (int k = 1; k < n_sl; ++k) CCNN_CUDA(cudaStreamWaitEvent(slots_[k].st, t0, 0));
    }
    // batched form: groups of batch_frames_ frames of one plan, each group one graph, the batch
    // contexts in turn (the next group is uploaded while the previous one runs); what is left over
    // (fewer frames than a group, or frames the batched form does not cover) runs frame by frame
    int first_single = 0;
    const int B = batch_frames_;
    if (B >= 2 && n_img >= B && inited_ && !batches_.empty()) {
        bool same = true;
        for (int i = 1; i < n_img && same; ++i)
            same = imgs[i].cols == imgs[0].cols && imgs[i].rows == imgs[0].rows && imgs[i].channels == imgs[0].channels;
        const Plan* p0 = nullptr;
        bool empty = false;
        if (same) {
            // admission of the first frame settles the detector's state (re-initialisation, and the
            // level count a first frame of the full size lowers, which keys a second, equal plan):
            // twice, so that every later admission of a frame of this size returns the same plan
            for (int rep = 0; rep < 2; ++rep) {
                ccnn_status st = prepare_frame(imgs[0], &p0, &empty);
                if (st != CCNN_OK) return st;
            }
        }
        if (same && !empty && inited_ && !batches_.empty() && batch_usable(*p0)) {
            const int n_full = n_img / B;
            const int n_ctx = (int)batches_.size();
            for (int g = 0; g < n_full; ++g) {
                BatchCtx& c = batches_[g % n_ctx];
                if (c.pending_first >= 0) {
                    ccnn_status st = collect_batch(c, B, faces, cap_per, n_faces, &worst);
                    if (st != CCNN_OK) return st;
                }
                for (int f = 0; f < B; ++f) {
                    const Plan* pf = nullptr;
                    ccnn_status st = prepare_frame(imgs[g * B + f], &pf, &empty);
                    if (st != CCNN_OK) return st;
                    if (pf != p0 || empty) {
                        set_error("internal: frames of one size gave different pyramid plans");
                        return CCNN_ERR_CUDA;
                    }
                }
                if (device_input) {
                    cudaStream_t cst = slots_[c.first_slot].st;
                    if (ordered_gen != init_gen_) {
                        CCNN_CUDA(cudaEventRecord(order_ev_, cudaStreamLegacy));
                        std::fill(waited.begin(), waited.end(), 0);
                        ordered_gen = init_gen_;
                    }
                    if (!waited[c.first_slot]) {
                        CCNN_CUDA(cudaStreamWaitEvent(cst, order_ev_, 0));
                        waited[c.first_slot] = 1;
                    }
                }
                ccnn_status st = launch_batch(c, *p0, imgs + (size_t)g * B, B, device_input);
                if (st != CCNN_OK) return st;
                c.pending_first = g * B;
            }
            for (auto& c : batches_)
                if (c.pending_first >= 0) {
                    ccnn_status st = collect_batch(c, B, faces, cap_per, n_faces, &worst);
                    if (st != CCNN_OK) return st;
                }
            first_single = n_full * B;
        }
    }
    for (int i = first_single; i < n_img; ++i) {
        const int k = i % n_sl;
        Slot& s = slots_[k];
        if (pending[k] >= 0) {
            ccnn_status st = collect(s, faces + (size_t)pending[k] * cap_per, cap_per, &n_faces[pending[k]]);
            if (st < 0) return st;
            if (st == CCNN_TRUNCATED) worst = CCNN_TRUNCATED;
            pending[k] = -1;
        }
        const Plan* p = nullptr;
        bool empty = false;
        // frame admission may re-initialise (and so free the slots): drain in-flight frames first
        if (!inited_ || imgs[i].cols > max_w_ || imgs[i].rows > max_h_ || (gray_image_only_ && input_downscale_ && imgs[i].channels != 1)) {
            for (int q = 0; q < n_sl; ++q)
                if (pending[q] >= 0) {
                    ccnn_status st = collect(slots_[q], faces + (size_t)pending[q] * cap_per, cap_per, &n_faces[pending[q]]);
                    if (st < 0) return st;
                    if (st == CCNN_TRUNCATED) worst = CCNN_TRUNCATED;
                    pending[q] = -1;
                }
        }
        ccnn_status st = prepare_frame(imgs[i], &p, &empty);
        if (st != CCNN_OK) return st;
        if (empty) {
            n_faces[i] = 0;
            continue;
        }
        if (device_input) {
            if (ordered_gen != init_gen_) {
                CCNN_CUDA(cudaEventRecord(order_ev_, cudaStreamLegacy));
                std::fill(waited.begin(), waited.end(), 0);
                ordered_gen = init_gen_;
            }
            if (!waited[k]) {
                CCNN_CUDA(cudaStreamWaitEvent(slots_[k].st, order_ev_, 0));
                waited[k] = 1;
            }
        }
        st = enqueue(slots_[k], *p, imgs[i], device_input, nullptr);
        if (st != CCNN_OK) return st;
        pending[k] = i;
    }
    if (t0) {
        if (inited_) {
            for (int k = 1; k < n_sl; ++k) CCNN_CUDA(cudaStreamWaitEvent(slots_[0].st, slots_[k].done, 0));
            CCNN_CUDA(cudaEventRecord(t1, slots_[0].st));
        }
    }
    for (int k = 0; k < n_sl; ++k)
        if (pending[k] >= 0) {
            ccnn_status st = collect(slots_[k], faces + (size_t)pending[k] * cap_per, cap_per, &n_faces[pending[k]]);
            if (st < 0) return st;
            if (st == CCNN_TRUNCATED) worst = CCNN_TRUNCATED;
        }
    if (t0) {
        float ms = 0.f;
        if (inited_ && cudaEventSynchronize(t1) == cudaSuccess && cudaEventElapsedTime(&ms, t0, t1) == cudaSuccess) *gpu_ms = ms;
        else *gpu_ms = -1.f;
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
    }
    return worst;
}

ccnn_status Detector::get_gray_device(const float** data, int* cols, int* rows, size_t* step) {
    std::lock_guard<std::mutex> lk(mu_);
    Slot& s = slots_[0];
    if (!inited_ || !s.last_plan) {
        set_error("no frame has been processed");
        return CCNN_ERR_INVALID_ARG;
    }
    *data = s.d_gray;
    *cols = s.last_plan->gw;
    *rows = s.last_plan->gh;
    *step = sizeof(float) * (size_t)s.gray_pitch;
    return CCNN_OK;
}

ccnn_status Detector::get_gray_host(float* out, int cap, int* cols, int* rows) {
    std::lock_guard<std::mutex> lk(mu_);
    Slot& s = slots_[0];
    if (!inited_ || !s.last_plan) {
        set_error("no frame has been processed");
        return CCNN_ERR_INVALID_ARG;
    }
    const Plan& p = *s.last_plan;
    *cols = p.gw;
    *rows = p.gh;
    if ((long long)p.gw * p.gh > cap) {
        set_error("output capacity too small");
        return CCNN_ERR_INVALID_ARG;
    }
    CCNN_CUDA(cudaMemcpy2D(out, sizeof(float) * p.gw, s.d_gray, sizeof(float) * s.gray_pitch, sizeof(float) * p.gw, p.gh,
                           cudaMemcpyDeviceToHost));
    return CCNN_OK;
}

ccnn_status Detector::get_params(ccnn_params* out) {
    std::lock_guard<std::mutex> lk(mu_);
    *out = api_;
    out->max_image_width = max_w_;
    out->max_image_height = max_h_;
    return CCNN_OK;
}

ccnn_status Detector::set_params(const ccnn_params& p) {
    std::lock_guard<std::mutex> lk(mu_);
    clear();
    api_ = p;
    max_w_ = p.max_image_width;
    max_h_ = p.max_image_height;
    gray_image_only_ = true;
    return CCNN_OK;  // the next frame re-initialises (Detect :2485-2492)
}

ccnn_status Detector::set_max_image_size(int w, int h) {
    std::lock_guard<std::mutex> lk(mu_);
    clear();
    max_w_ = w;
    max_h_ = h;
    return CCNN_OK;
}

ccnn_status Detector::set_min_object_height(int v) {
    std::lock_guard<std::mutex> lk(mu_);
    clear();
    api_.min_face_height = v;
    return CCNN_OK;
}

ccnn_status Detector::set_max_object_height(int v) {
    std::lock_guard<std::mutex> lk(mu_);
    clear();
    api_.max_face_height = v;
    return CCNN_OK;
}

ccnn_status Detector::set_num_threads(int v) {
    std::lock_guard<std::mutex> lk(mu_);
    api_.num_threads = v;  // the cascade's parallelism is on the device; kept for getParam
    return CCNN_OK;
}

ccnn_status Detector::stage1_forward(const float* d_img, int w, int h, size_t step, float* d_resp, int cap, int* rw, int* rh,
                                     cudaStream_t st) {
    std::lock_guard<std::mutex> lk(mu_);
    if (!inited_) {
        ccnn_status s = init();
        if (s != CCNN_OK) return s;
    }
    if (w < pat_w_ || h < pat_h_ || (step % sizeof(float)) != 0) {
        set_error("image smaller than the stage-1 window or misaligned step");
        return CCNN_ERR_INVALID_ARG;
    }
    if (legacy_) {
        set_error("stage-1 inspection covers the CNTK family; use ccnn_legacy_net_forward for legacy models");
        return CCNN_ERR_UNSUPPORTED;
    }
    cudaSetDevice(device_);
    LevelDesc L{};
    L.w = w;
    L.h = h;
    L.mode = 0;
    L.scale = 1.f;
    L.inv_scale = 1.f;
    L.p1w = (w - 3) >> 1;
    L.p1h = (h - 3) >> 1;
    L.p2w = (L.p1w - 2) >> 1;
    L.p2h = (L.p1h - 2) >> 1;
    L.ow = L.p2w - 3;
    L.oh = L.p2h - 4;
    L.s1_pitch = (int)round_up(L.p1w, 32);
    L.s1_plane = (long long)L.s1_pitch * L.p1h;
    L.k1_tiles_x = (L.p1w + kK1TileX - 1) / kK1TileX;
    L.k2_tiles_x = (L.ow + kK2TileX - 1) / kK2TileX;
    L.img_pitch = (int)(step / sizeof(float));
    L.img_vec = (L.img_pitch % 4 == 0 && (reinterpret_cast<uintptr_t>(d_img) & 15) == 0) ? 1 : 0;
    *rw = L.ow;
    *rh = L.oh;
    if ((long long)L.ow * L.oh > cap) {
        set_error("response capacity too small");
        return CCNN_ERR_INVALID_ARG;
    }
    float* d_s1 = nullptr;
    CCNN_CUDA(cudaMallocAsync(&d_s1, sizeof(float) * 4 * L.s1_plane, st));
    CCNN_CUDA(launch_stage1(w1_, &L, 1, d_img, d_s1, d_resp, st));
    CCNN_CUDA(cudaFreeAsync(d_s1, st));
    CCNN_CUDA(cudaStreamSynchronize(st));
    return CCNN_OK;
}

// Re-runs the last frame's kernel chain on slot 0 `iters` times with an event between every
// two kernels; ms[k] gets the mean duration of kernel k: gray, pyramid (legacy family only: the CNTK
// front kernel resamples the levels itself, so this entry is the empty gap), stage-1 front, stage-1
// back (with the candidate count and the memset of the counts before it), candidate write,
// stage-2/3 windows, replay; ms[7] the learned gate; ms[8] the pyramid and stage 1 as one
// persistent launch.
ccnn_status Detector::profile(int iters, float* ms, int n_ms) {
    std::lock_guard<std::mutex> lk(mu_);
    Slot& s = slots_[0];
    if (!inited_ || !s.last_plan || iters <= 0) {
        set_error("no frame has been processed");
        return CCNN_ERR_INVALID_ARG;
    }
    if (s.last_in_place) {
        // the last frame was read from the caller's device memory, which may be gone by now
        set_error("the last frame was read in place from device memory; profile a frame given from host memory");
        return CCNN_ERR_UNSUPPORTED;
    }
    cudaSetDevice(device_);
    const Plan& p = *s.last_plan;
    constexpr int K = 7;
    cudaEvent_t ev[K + 2];  // ev[K + 1]: end of the learned gate, when it runs
    for (auto& e : ev) CCNN_CUDA(cudaEventCreate(&e));
    double acc[K + 1] = {0};
    const bool gated = gate_on_ && s.gate.prob && p.gw >= 32 && p.gh >= 32;
    const ReplayArgs a = replay_args(s, p);
    for (int it = 0; it < iters; ++it) {
        CCNN_CUDA(cudaEventRecord(ev[0], s.st));
        __half* feat = (gated && !p.downscale) ? s.gate.feat : nullptr;
        if (p.downscale)
            CCNN_CUDA(launch_gray_u8_resized(s.d_in, (int)p.in_pitch, p.in_w, p.in_h, s.d_gray, s.gray_pitch, p.gw, p.gh, s.st));
        else
            CCNN_CUDA(launch_gray(s.d_in, (int)p.in_pitch, p.in_w, p.in_h, p.ch, s.d_gray, s.gray_pitch, s.st, feat));
        CCNN_CUDA(cudaEventRecord(ev[1], s.st));
        if (gated) {
            CCNN_CUDA(launch_gate(gate_net_, s.d_gray, s.gray_pitch, p.gw, p.gh, feat != nullptr, p.levels.data(), p.n_levels, s.gate, gate_thr_,
                                  gate_amb_frac_, gate_margin_, s.d_back_on, s.d_front_on, s.st));
        }
        CCNN_CUDA(cudaEventRecord(ev[K + 1], s.st));
        if (legacy_) CCNN_CUDA(launch_pyramid(p.levels.data(), p.n_levels, s.d_gray, s.gray_pitch, p.gw, p.gh, s.d_limg, s.st));
        CCNN_CUDA(cudaEventRecord(ev[2], s.st));
        if (!legacy_)
            CCNN_CUDA(launch_stage1_front(w1_, p.levels.data(), p.n_levels, nullptr, s.d_s1, s.st, gated ? s.d_front_on : nullptr, s1_sched_,
                                          GrayRef{s.d_gray, s.gray_pitch, p.gw, p.gh}));
        CCNN_CUDA(cudaEventRecord(ev[3], s.st));
        if (!p.chunks.empty()) CCNN_CUDA(cudaMemsetAsync(s.d_counts, 0, sizeof(int) * p.chunks.size(), s.st));
        if (legacy_) {  // the legacy network's three layers all count as the back entry
            const ccnn_status ls = enqueue_legacy_stage1(s, p);
            if (ls != CCNN_OK) return ls;
        } else
            CCNN_CUDA(launch_stage1_back(w1_, p.levels.data(), p.n_levels, s.d_s1, s.d_resp, s.st, s.d_counts, cfg_.thr1,
                                         gated ? s.d_back_on : nullptr, gated ? gate_cells(s.gate, p.gw, p.gh, gate_amb_frac_, gate_margin_) : GateCells{},
                                         s1_sched_));
        CCNN_CUDA(cudaEventRecord(ev[4], s.st));
        CCNN_CUDA(launch_cand_write(p.d_chunks, (int)p.chunks.size(), p.d_levels, s.d_resp, cfg_.thr1, s.d_counts, s.d_cands, s.d_ncand,
                                    (int)cand_cap_, s.st));
        CCNN_CUDA(cudaEventRecord(ev[5], s.st));
        if (detect_enabled_)
            CCNN_CUDA(launch_window(*wn_, s.d_gray, s.gray_pitch, p.gw, p.gh, s.d_cands, s.d_ncand, p.d_levels, s.d_win, cfg_,
                                    window_grid_, s.st, legacy_ ? d_lg_ : nullptr, window_ctas_per_sm_));
        if (s.d_attr)
            CCNN_CUDA(launch_facial(d_lnet_, s.d_gray, s.gray_pitch, p.gw, p.gh, s.d_cands, s.d_ncand, p.d_levels, s.d_win, cfg_,
                                    s.d_attr, facial_grid_, s.st));
        CCNN_CUDA(cudaEventRecord(ev[6], s.st));
        CCNN_CUDA(launch_replay(a, s.st));
        CCNN_CUDA(cudaEventRecord(ev[7], s.st));
        CCNN_CUDA(cudaEventSynchronize(ev[7]));
        for (int k = 0; k < K; ++k) {
            float m = 0.f;
            CCNN_CUDA(cudaEventElapsedTime(&m, k == 1 ? ev[K + 1] : ev[k], ev[k + 1]));
            acc[k] += m;
        }
        float m = 0.f;
        CCNN_CUDA(cudaEventElapsedTime(&m, ev[1], ev[K + 1]));
        acc[K] += m;
    }
    // entry K + 1: the pyramid and stage 1 of the frame as one persistent launch (the batched form's
    // kernel on this frame), measured the same way
    double single = 0.0;
    if (n_ms > K + 1 && !legacy_ && p.n_levels > 0 && p.n_levels <= kMaxBatchLevels) {
        BatchFrames F{};
        F.gray[0] = s.d_gray;
        F.gpitch = s.gray_pitch;
        F.gw = p.gw;
        F.gh = p.gh;
        F.s1[0] = s.d_s1;
        F.resp[0] = s.d_resp;
        F.counts[0] = s.d_counts;
        F.front_on[0] = gated ? s.d_front_on : nullptr;
        F.back_on[0] = gated ? s.d_back_on : nullptr;
        F.cells[0] = gated ? gate_cells(s.gate, p.gw, p.gh, gate_amb_frac_, gate_margin_) : GateCells{};
        BatchQueue Q;
        build_batch_queue(&Q, 1, p.n_levels, (int)p.chunks.size(), p.k1_tiles, p.k2_tiles, cfg_.thr1);
        const int grid = sm_count_ * stage1_batch_blocks_per_sm(batch_bpsm_);
        for (int it = 0; it < iters; ++it) {
            CCNN_CUDA(cudaMemsetAsync(s.d_sync1, 0, sizeof(int) * (2 + kBatchStages), s.st));
            if (!p.chunks.empty()) CCNN_CUDA(cudaMemsetAsync(s.d_counts, 0, sizeof(int) * p.chunks.size(), s.st));
            CCNN_CUDA(cudaEventRecord(ev[0], s.st));
            CCNN_CUDA(launch_stage1_batch(w1_, F, Q, p.d_levels, s.d_sync1, s.d_sync1 + 1 + kBatchStages, grid, s.st, batch_bpsm_));
            CCNN_CUDA(cudaEventRecord(ev[1], s.st));
            CCNN_CUDA(cudaEventSynchronize(ev[1]));
            float m = 0.f;
            CCNN_CUDA(cudaEventElapsedTime(&m, ev[0], ev[1]));
            single += m;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int k = 0; k < n_ms && k < K + 1; ++k) ms[k] = (float)(acc[k] / iters);
    if (n_ms > K + 1) ms[K + 1] = (float)(single / iters);
    return CCNN_OK;
}

ccnn_status Detector::inspect_levels(ccnn_level_info* out, int cap, int* n) {
    std::lock_guard<std::mutex> lk(mu_);
    const Plan* p = slots_[0].last_plan;
    if (!inited_ || !p) {
        set_error("no frame has been processed");
        return CCNN_ERR_INVALID_ARG;
    }
    *n = p->n_levels;
    for (int i = 0; i < p->n_levels && i < cap; ++i) {
        const LevelDesc& L = p->levels[i];
        out[i].width = L.w;
        out[i].height = L.h;
        out[i].scale = L.scale;
        out[i].resp_width = L.ow;
        out[i].resp_height = L.oh;
    }
    return CCNN_OK;
}

ccnn_status Detector::inspect_response(int level, float* out, int cap) {
    std::lock_guard<std::mutex> lk(mu_);
    const Plan* p = slots_[0].last_plan;
    if (!inited_ || !p || level < 0 || level >= p->n_levels) {
        set_error("no such level");
        return CCNN_ERR_INVALID_ARG;
    }
    const LevelDesc& L = p->levels[level];
    if ((long long)L.ow * L.oh > cap) {
        set_error("output capacity too small");
        return CCNN_ERR_INVALID_ARG;
    }
    CCNN_CUDA(cudaMemcpy(out, slots_[0].d_resp + L.resp_off, sizeof(float) * L.ow * L.oh, cudaMemcpyDeviceToHost));
    return CCNN_OK;
}

ccnn_status Detector::inspect_candidates(ccnn_candidate* out, int cap, int* n) {
    std::lock_guard<std::mutex> lk(mu_);
    Slot& s = slots_[0];
    if (!inited_ || !s.last_plan) {
        set_error("no frame has been processed");
        return CCNN_ERR_INVALID_ARG;
    }
    int nc = 0;
    CCNN_CUDA(cudaMemcpy(&nc, s.d_ncand, sizeof(int), cudaMemcpyDeviceToHost));
    *n = nc;
    const int take = std::min(nc, cap);
    std::vector<Candidate> c(take);
    std::vector<CandResult> r(take);
    if (take > 0) {
        CCNN_CUDA(cudaMemcpy(c.data(), s.d_cands, sizeof(Candidate) * take, cudaMemcpyDeviceToHost));
        if (detect_enabled_) CCNN_CUDA(cudaMemcpy(r.data(), s.d_results, sizeof(CandResult) * take, cudaMemcpyDeviceToHost));
    }
    for (int i = 0; i < take; ++i) {
        out[i].level = c[i].level;
        out[i].x = c[i].px;
        out[i].y = c[i].py;
        out[i].score = c[i].score;
        out[i].accepted = detect_enabled_ ? r[i].accepted : 0;
        out[i].check_score = detect_enabled_ ? r[i].score : 0.f;
        out[i].knn = detect_enabled_ ? r[i].knn : 0;
    }
    return CCNN_OK;
}

ccnn_status Detector::inspect_raw(ccnn_detection* out, int cap, int* n) {
    std::lock_guard<std::mutex> lk(mu_);
    Slot& s = slots_[0];
    if (!inited_ || !s.last_plan) {
        set_error("no frame has been processed");
        return CCNN_ERR_INVALID_ARG;
    }
    int nr = 0;
    CCNN_CUDA(cudaMemcpy(&nr, s.d_nraw, sizeof(int), cudaMemcpyDeviceToHost));
    *n = nr;
    const int take = std::min(nr, cap);
    std::vector<Det> d(take);
    if (take > 0) CCNN_CUDA(cudaMemcpy(d.data(), s.D, sizeof(Det) * take, cudaMemcpyDeviceToHost));
    for (int i = 0; i < take; ++i) {
        out[i].x = d[i].x;
        out[i].y = d[i].y;
        out[i].width = d[i].w;
        out[i].height = d[i].h;
        out[i].score = d[i].score;
        out[i].scale = d[i].scale;
        out[i].knn = d[i].knn;
        out[i].num_detect = d[i].num_detect;
    }
    return CCNN_OK;
}

// ---------------- batched form: groups of B frames in one graph ----------------

ccnn_status Detector::alloc_batches() {
    batches_.clear();
    const int B = batch_frames_;
    if (B < 2 || (int)slots_.size() < B) return CCNN_OK;
    const int n_ctx = (int)slots_.size() / B;
    batches_.assign(n_ctx, BatchCtx());
    const long long face_cap = std::max<long long>(cand_cap_, kHostFaces);
    for (int k = 0; k < n_ctx; ++k) {
        BatchCtx& c = batches_[k];
        c.first_slot = k * B;
        CCNN_CUDA(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming));
        CCNN_CUDA(cudaMalloc(&c.d_sync, sizeof(int) * (2 + kBatchStages * B)));
        CCNN_CUDA(cudaMalloc(&c.d_rargs, sizeof(ReplayArgs) * B));
        CCNN_CUDA(cudaMalloc(&c.d_src, sizeof(FrameSrc) * B));
        CCNN_CUDA(cudaMallocHost(&c.h_src, sizeof(FrameSrc) * B));
        CCNN_CUDA(cudaMalloc(&c.d_faces, sizeof(FaceOut) * face_cap * B));
        CCNN_CUDA(cudaMalloc(&c.d_nf, sizeof(int) * B));
        CCNN_CUDA(cudaMallocHost(&c.h_faces, sizeof(FaceOut) * kGraphFaces * B));
        CCNN_CUDA(cudaMallocHost(&c.h_nf, sizeof(int) * (B + 1)));
    }
    return CCNN_OK;
}

void Detector::free_batches() {
    for (auto& c : batches_) {
        if (c.done) cudaEventSynchronize(c.done);
        if (c.exec) cudaGraphExecDestroy(c.exec);
        cudaFree(c.d_sync);
        cudaFree(c.d_rargs);
        cudaFree(c.d_src);
        cudaFreeHost(c.h_src);
        cudaFree(c.d_faces);
        cudaFree(c.d_nf);
        cudaFreeHost(c.h_faces);
        cudaFreeHost(c.h_nf);
        if (c.done) cudaEventDestroy(c.done);
    }
    batches_.clear();
}

// The batched form covers the CNTK cascade on frames at their own resolution (no input downscale),
// without facial analysis; other configurations run every frame as its own graph.
// One persistent launch for the pyramid and stage 1 of a frame: the schedule's batch_frames == 1,
// or AdvancedParam::packet_detection on a GPU pipeline (the reference's CUDA build keeps packet mode
// only there, cnn_detector_v3.cpp:67-84; precision `def` turns it off, :922-925). CNTK cascade only.
bool Detector::single_launch_stage1() const {
    if (legacy_) return false;
    const bool packet = has_cnn_ && cnn_ap_.packet_detection && cnn_p_.pipeline != CCNN_PIPELINE_CPU &&
                        cnn_ap_.detect_precision != CCNN_PRECISION_DEF;
    return batch_frames_ == 1 || packet;
}

bool Detector::batch_usable(const Plan& p) const {
    return !batches_.empty() && !legacy_ && !d_lnet_ && !p.downscale && p.n_levels > 0 && p.n_levels <= kMaxBatchLevels &&
           (p.ch == 1 || p.ch == 3 || p.ch == 4);
}

// The graph of a batch: gray of every frame in one launch, the learned gate per frame (when on), the
// pyramid and stage 1 of every level of every frame in one persistent launch fed by a device work
// queue (front items resample their level tiles from the gray frames), the candidates of every frame in one launch, the
// stage-2/3 windows of every frame's candidates in one persistent launch, every frame's replay in one
// launch (a block each), then the results to the host.
ccnn_status Detector::enqueue_batch_kernels(BatchCtx& c, const Plan& p, int B) {
    cudaStream_t st = slots_[c.first_slot].st;
    const bool gated = gate_on_ && slots_[c.first_slot].gate.prob && p.gw >= 32 && p.gh >= 32;
    BatchFrames F{};
    BatchCands C{};
    WinBatch WB{};
    WB.n_frames = B;
    for (int f = 0; f < B; ++f) {
        Slot& s = slots_[c.first_slot + f];
        F.gray[f] = s.d_gray;
        F.feat[f] = gated ? s.gate.feat : nullptr;
        F.s1[f] = s.d_s1;
        F.resp[f] = s.d_resp;
        F.counts[f] = s.d_counts;
        F.front_on[f] = gated ? s.d_front_on : nullptr;
        F.back_on[f] = gated ? s.d_back_on : nullptr;
        F.cells[f] = gated ? gate_cells(s.gate, p.gw, p.gh, gate_amb_frac_, gate_margin_) : GateCells{};
        C.cands[f] = s.d_cands;
        C.ncand[f] = s.d_ncand;
        WB.gray[f] = s.d_gray;
        WB.cands[f] = s.d_cands;
        WB.ncand[f] = s.d_ncand;
        WB.out[f] = s.d_win;
    }
    const int gpitch = slots_[c.first_slot].gray_pitch;
    F.gpitch = gpitch;
    F.gw = p.gw;
    F.gh = p.gh;
    CCNN_CUDA(cudaMemsetAsync(c.d_sync, 0, sizeof(int) * (2 + kBatchStages * B), st));
    CCNN_CUDA(launch_gray_batch(c.d_src, B, p.in_w, p.in_h, p.ch, F, gpitch, st));
    if (gated)
        for (int f = 0; f < B; ++f) {
            Slot& s = slots_[c.first_slot + f];
            CCNN_CUDA(launch_gate(gate_net_, s.d_gray, s.gray_pitch, p.gw, p.gh, true, p.levels.data(), p.n_levels, s.gate, gate_thr_,
                                  gate_amb_frac_, gate_margin_, s.d_back_on, s.d_front_on, st));
        }
    CCNN_CUDA(launch_counts_zero_batch(F, (int)p.chunks.size(), B, st));
    BatchQueue Q;
    build_batch_queue(&Q, B, p.n_levels, (int)p.chunks.size(), p.k1_tiles, p.k2_tiles, cfg_.thr1);
    const int grid = sm_count_ * stage1_batch_blocks_per_sm(batch_bpsm_);
    int* sync = c.d_sync;
    int* err = c.d_sync + 1 + kBatchStages * B;
    CCNN_CUDA(launch_stage1_batch(w1_, F, Q, p.d_levels, sync, err, grid, st, batch_bpsm_));
    CCNN_CUDA(launch_cand_write_batch(p.d_chunks, (int)p.chunks.size(), p.d_levels, F, C, B, cfg_.thr1, (int)cand_cap_, st));
    if (detect_enabled_) CCNN_CUDA(launch_window_batch(*wn_, WB, gpitch, p.gw, p.gh, p.d_levels, cfg_, window_grid_, st, window_ctas_per_sm_));
    CCNN_CUDA(launch_replay_batch(c.d_rargs, B, st));
    const long long face_cap = std::max<long long>(cand_cap_, kHostFaces);
    CCNN_CUDA(cudaMemcpyAsync(c.h_nf, c.d_nf, sizeof(int) * B, cudaMemcpyDeviceToHost, st));
    CCNN_CUDA(cudaMemcpyAsync(c.h_nf + B, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CCNN_CUDA(cudaMemcpy2DAsync(c.h_faces, sizeof(FaceOut) * kGraphFaces, c.d_faces, sizeof(FaceOut) * face_cap, sizeof(FaceOut) * kGraphFaces, B,
                                cudaMemcpyDeviceToHost, st));
    return CCNN_OK;
}

ccnn_status Detector::launch_batch(BatchCtx& c, const Plan& p, const ccnn_image* imgs, int B, bool device_input) {
    cudaStream_t st = slots_[c.first_slot].st;
    const bool gated = gate_on_ && slots_[c.first_slot].gate.prob && p.gw >= 32 && p.gh >= 32;
    if (c.exec_plan != &p || c.exec_gated != gated) {
        if (c.exec) {
            cudaGraphExecDestroy(c.exec);
            c.exec = nullptr;
        }
        // per-frame replay arguments of this plan (device memory the replay kernel reads)
        const long long face_cap = std::max<long long>(cand_cap_, kHostFaces);
        std::vector<ReplayArgs> ra(B);
        for (int f = 0; f < B; ++f) {
            ra[f] = replay_args(slots_[c.first_slot + f], p);
            ra[f].faces = c.d_faces + (size_t)f * face_cap;
            ra[f].face_cap = (int)face_cap;
            ra[f].n_faces = c.d_nf + f;
        }
        CCNN_CUDA(cudaMemcpyAsync(c.d_rargs, ra.data(), sizeof(ReplayArgs) * B, cudaMemcpyHostToDevice, st));
        CCNN_CUDA(cudaStreamSynchronize(st));
        cudaGraph_t g;
        CCNN_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        ccnn_status es = enqueue_batch_kernels(c, p, B);
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        if (es != CCNN_OK) return es;
        CCNN_CUDA(ce);
        ce = cudaGraphInstantiate(&c.exec, g, 0);
        cudaGraphDestroy(g);
        CCNN_CUDA(ce);
        c.exec_plan = &p;
        c.exec_gated = gated;
    }
    // sources: aligned device frames are read where they are; others are packed into the slot
    for (int f = 0; f < B; ++f) {
        const ccnn_image& img = imgs[f];
        Slot& s = slots_[c.first_slot + f];
        const bool in_place = device_input && !((uintptr_t)img.data & 63) && !(img.step & 63) && img.step <= (size_t)INT32_MAX;
        if (in_place) {
            c.h_src[f].data = img.data;
            c.h_src[f].pitch = (int)img.step;
        } else {
            const size_t row = (size_t)img.cols * img.channels;
            const cudaMemcpyKind kind = device_input ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
            if (img.step == p.in_pitch)
                CCNN_CUDA(cudaMemcpyAsync(s.d_in, img.data, p.in_pitch * (size_t)(img.rows - 1) + row, kind, st));
            else
                CCNN_CUDA(cudaMemcpy2DAsync(s.d_in, p.in_pitch, img.data, img.step, row, img.rows, kind, st));
            c.h_src[f].data = s.d_in;
            c.h_src[f].pitch = (int)p.in_pitch;
        }
        c.h_src[f].pad = 0;
        s.last_in_place = in_place;
        s.last_plan = &p;
    }
    CCNN_CUDA(cudaMemcpyAsync(c.d_src, c.h_src, sizeof(FrameSrc) * B, cudaMemcpyHostToDevice, st));
    CCNN_CUDA(cudaGraphLaunch(c.exec, st));
    CCNN_CUDA(cudaEventRecord(c.done, st));
    CCNN_CUDA(cudaEventRecord(slots_[c.first_slot].done, st));
    return CCNN_OK;
}

ccnn_status Detector::collect_batch(BatchCtx& c, int B, ccnn_face* faces, int cap_per, int* n_faces, ccnn_status* worst) {
    CCNN_CUDA(cudaEventSynchronize(c.done));
    CCNN_CUDA(cudaGetLastError());
    if (c.h_nf[B] != 0) {
        set_error("batched stage 1: a dependency wait gave up (results of the batch discarded)");
        return CCNN_ERR_CUDA;
    }
    const long long face_cap = std::max<long long>(cand_cap_, kHostFaces);
    for (int f = 0; f < B; ++f) {
        const int img = c.pending_first + f;
        const int nf = c.h_nf[f];
        const int take = std::min(nf, cap_per);
        const FaceOut* src = c.h_faces + (size_t)f * kGraphFaces;
        if (take > kGraphFaces) {
            c.h_extra.resize(take);
            CCNN_CUDA(cudaMemcpy(c.h_extra.data(), c.d_faces + (size_t)f * face_cap, sizeof(FaceOut) * take, cudaMemcpyDeviceToHost));
            src = c.h_extra.data();
        }
        ccnn_face* out = faces + (size_t)img * cap_per;
        for (int i = 0; i < take; ++i) {
            out[i].x = src[i].x;
            out[i].y = src[i].y;
            out[i].width = src[i].w;
            out[i].height = src[i].h;
            out[i].score = src[i].score;
            out[i].gender = src[i].gender;
            out[i].smile = src[i].smile;
            out[i].glasses = src[i].glasses;
        }
        n_faces[img] = nf;
        if (nf > cap_per) *worst = CCNN_TRUNCATED;
    }
    c.pending_first = -1;
    return CCNN_OK;
}

// ---------------- the internal CNNDetector class (cnn_detector_v3.h:82-453) ----------------

// CNNDetector::Param + AdvancedParam -> the FaceDetector-shaped parameters the rest of the detector
// reads (the inverse of paramConverter, CompactCNNLibAPI_v2.cpp:51-88).
void Detector::cnn_to_api() {
    ccnn_default_params(&api_);
    api_.max_image_width = cnn_p_.max_image_width;
    api_.max_image_height = cnn_p_.max_image_height;
    api_.min_face_height = cnn_p_.min_obj_height;
    api_.max_face_height = cnn_p_.max_obj_height;
    api_.scale_factor = cnn_p_.scale_factor;
    api_.min_neighbors = cnn_p_.min_neighbors;
    api_.num_threads = cnn_p_.num_threads;
    api_.pipeline = cnn_p_.pipeline;
    api_.detect_precision = cnn_ap_.detect_precision;
    api_.treshold[0] = cnn_ap_.treshold_1;
    api_.treshold[1] = cnn_ap_.treshold_2;
    api_.treshold[2] = cnn_ap_.treshold_3;
    api_.drop_detect = cnn_ap_.drop_detect;
    api_.equalize = cnn_ap_.equalize;
    api_.reflection = cnn_ap_.reflection;
    api_.detect_mode = cnn_ap_.detect_mode;
    for (int i = 0; i < 3; ++i) api_.index_output[i] = cnn_ap_.index_output[i];
    api_.device_info = cnn_ap_.device_info;
    api_.cuda_device_id = cnn_ap_.cuda_device_id;
    api_.cl_platform_id = cnn_ap_.cl_platform_id;
    api_.cl_device_id = cnn_ap_.cl_device_id;
    api_.facial_analysis = cnn_ap_.facial_analysis;
}

static ccnn_status check_cnn_params(const ccnn_cnn_advanced_param& ap) {
    if (ap.blur || ap.uniform_noise) {
        // CNNDetector::Init resets both only for precision `def`; the reference's CPU path never reads
        // blur, and uniform_noise draws from std::rand, which no parity contract can pin
        if (ap.detect_precision != CCNN_PRECISION_DEF) {
            set_error("AdvancedParam: blur and uniform_noise are not supported");
            return CCNN_ERR_UNSUPPORTED;
        }
    }
    return CCNN_OK;
}

ccnn_status Detector::create_cnn(const ccnn_cnn_param& p, const ccnn_cnn_advanced_param& ap, const char* const* model_paths) {
    const ccnn_status cs = check_cnn_params(ap);
    if (cs != CCNN_OK) return cs;
    has_cnn_ = true;
    cnn_p_ = p;
    cnn_ap_ = ap;
    cnn_to_api();
    slots_.assign(1, Slot());  // Detect is synchronous: one frame slot
    for (int i = 0; i < 3; ++i) {
        const char* mp = model_paths ? model_paths[i] : nullptr;
        static const char* kNames[3] = {"cnn4face1_cntk.bin", "cnn4face2_cntk.bin", "cnn4face3_cntk.bin"};
        model_paths_[i] = (mp && mp[0]) ? std::string(mp) : bundled_model_dir() + "/" + kNames[i];
    }
    gray_image_only_ = ap.gray_image_only != 0;
    max_w_ = p.max_image_width;
    max_h_ = p.max_image_height;
    return init();
}

static Det det_from(const ccnn_detection& d) {
    Det r;
    r.x = d.x;
    r.y = d.y;
    r.w = d.width;
    r.h = d.height;
    r.x2 = d.x + d.width;
    r.y2 = d.y + d.height;
    r.score = d.score;
    r.scale = d.scale;
    r.knn = d.knn;
    r.num_detect = d.num_detect;
    return r;
}

static ccnn_detection detection_from(const Det& d) {
    ccnn_detection r;
    r.x = d.x;
    r.y = d.y;
    r.width = d.w;
    r.height = d.h;
    r.score = d.score;
    r.scale = d.scale;
    r.knn = d.knn;
    r.num_detect = d.num_detect;
    return r;
}

ccnn_status Detector::detect_cnn(const ccnn_image& img, const ccnn_detection* prior, int n_prior, ccnn_detection* out, int cap, int* n) {
    std::lock_guard<std::mutex> lk(mu_);
    if (!n || cap < 0 || (cap > 0 && !out) || n_prior < 0 || (n_prior > 0 && !prior)) {
        set_error("invalid output arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    cudaSetDevice(device_);
    std::vector<ccnn_detection> keep(prior, prior + n_prior);  // `prior` may alias `out`
    auto give = [&](const std::vector<ccnn_detection>& v) {
        *n = (int)v.size();
        for (int i = 0; i < (int)v.size() && i < cap; ++i) out[i] = v[i];
        return (int)v.size() > cap ? CCNN_TRUNCATED : CCNN_OK;
    };
    const Plan* p = nullptr;
    bool empty = false;
    ccnn_status st = prepare_frame(img, &p, &empty);
    if (st != CCNN_OK) return st;
    if (empty) return give(keep);  // a frame smaller than the check window: detections untouched (:2494-2497)
    Slot& s = slots_[0];
    st = enqueue(s, *p, img, false, nullptr);
    if (st != CCNN_OK) return st;
    int nf = 0;
    const FaceOut* src = nullptr;
    st = collect_raw(s, (int)std::min<long long>(std::max<long long>(cand_cap_, kHostFaces), INT32_MAX), &nf, &src);
    if (st != CCNN_OK) return st;
    std::vector<ccnn_detection> res;
    if (n_prior == 0 || !merger_detect_) {
        // the priors are dropped when the raw list is copied out unmerged (:2775-2779)
        int nraw = 0;
        if (n_prior > 0) CCNN_CUDA(cudaMemcpy(&nraw, s.d_nraw, sizeof(int), cudaMemcpyDeviceToHost));
        if (n_prior > 0 && nraw == 0) return give(keep);
        res.resize(nf);
        for (int i = 0; i < nf; ++i) {
            res[i].x = src[i].x;
            res[i].y = src[i].y;
            res[i].width = src[i].w;
            res[i].height = src[i].h;
            res[i].score = src[i].score;
            res[i].scale = src[i].scale;
            res[i].knn = src[i].knn;
            res[i].num_detect = src[i].num_detect;
        }
        return give(res);
    }
    int nraw = 0;
    CCNN_CUDA(cudaMemcpy(&nraw, s.d_nraw, sizeof(int), cudaMemcpyDeviceToHost));
    if (nraw == 0) return give(keep);  // no new raw detection: the vector is left as it was (:2749)
    int nmk = 0;
    CCNN_CUDA(cudaMemcpy(&nmk, s.d_nmk, sizeof(int), cudaMemcpyDeviceToHost));
    // [priors, new clusters] -> filter -> Merger(0.2, del) -> rescale, on the device
    const int total = n_prior + nmk;
    std::vector<Det> h_prior(n_prior);
    for (int i = 0; i < n_prior; ++i) h_prior[i] = det_from(keep[i]);
    Det *d_prior = nullptr, *d_list = nullptr, *d_out = nullptr;
    uint8_t* d_checked = nullptr;
    int* d_n = nullptr;
    cudaError_t e = cudaMallocAsync(&d_prior, sizeof(Det) * n_prior, s.st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_list, sizeof(Det) * 2 * (size_t)total, s.st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_out, sizeof(Det) * (size_t)total, s.st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_checked, (size_t)total, s.st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_n, sizeof(int), s.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_prior, h_prior.data(), sizeof(Det) * n_prior, cudaMemcpyHostToDevice, s.st);
    if (e == cudaSuccess) e = launch_prior_merge(d_prior, n_prior, s.d_mk, s.d_nmk, cfg_, d_list, d_checked, d_out, d_n, s.st);
    int nout = 0;
    std::vector<Det> h_out((size_t)total);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nout, d_n, sizeof(int), cudaMemcpyDeviceToHost, s.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_out.data(), d_out, sizeof(Det) * (size_t)total, cudaMemcpyDeviceToHost, s.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.st);
    for (void* q : {(void*)d_prior, (void*)d_list, (void*)d_out, (void*)d_checked, (void*)d_n})
        if (q) cudaFreeAsync(q, s.st);
    CCNN_CUDA(e);
    CCNN_CUDA(cudaStreamSynchronize(s.st));
    if (nout == 0 && total == 0) return give(keep);
    res.resize(nout);
    for (int i = 0; i < nout; ++i) res[i] = detection_from(h_out[i]);
    return give(res);
}

ccnn_status Detector::nms(const ccnn_detection* rect, int n_rect, ccnn_detection* out, int cap, int* n_out) {
    std::lock_guard<std::mutex> lk(mu_);
    if (!n_out || n_rect < 0 || (n_rect > 0 && !rect) || cap < 0 || (cap > 0 && !out)) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    *n_out = 0;
    if (n_rect == 0) return CCNN_OK;
    if (!inited_) {
        ccnn_status st = init();
        if (st != CCNN_OK) return st;
    }
    cudaSetDevice(device_);
    Slot& s = slots_[0];
    std::vector<Det> h_in(n_rect);
    for (int i = 0; i < n_rect; ++i) h_in[i] = det_from(rect[i]);
    Det *d_in = nullptr, *d_out = nullptr;
    uint8_t* d_checked = nullptr;
    int* d_n = nullptr;
    cudaError_t e = cudaMallocAsync(&d_in, sizeof(Det) * n_rect, s.st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_out, sizeof(Det) * n_rect, s.st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_checked, n_rect, s.st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_n, sizeof(int), s.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_in, h_in.data(), sizeof(Det) * n_rect, cudaMemcpyHostToDevice, s.st);
    if (e == cudaSuccess) e = launch_nms(d_in, n_rect, d_checked, d_out, d_n, s.st);
    int nout = 0;
    std::vector<Det> h_out(n_rect);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nout, d_n, sizeof(int), cudaMemcpyDeviceToHost, s.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_out.data(), d_out, sizeof(Det) * n_rect, cudaMemcpyDeviceToHost, s.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.st);
    for (void* q : {(void*)d_in, (void*)d_out, (void*)d_checked, (void*)d_n})
        if (q) cudaFreeAsync(q, s.st);
    CCNN_CUDA(e);
    CCNN_CUDA(cudaStreamSynchronize(s.st));
    *n_out = nout;
    for (int i = 0; i < nout && i < cap; ++i) out[i] = detection_from(h_out[i]);
    return nout > cap ? CCNN_TRUNCATED : CCNN_OK;
}

ccnn_status Detector::get_cnn_params(ccnn_cnn_param* p, ccnn_cnn_advanced_param* ap) {
    std::lock_guard<std::mutex> lk(mu_);
    if (!has_cnn_) {
        set_error("the handle was not created through the CNNDetector API");
        return CCNN_ERR_INVALID_ARG;
    }
    if (p) {
        *p = cnn_p_;
        p->max_image_width = max_w_;
        p->max_image_height = max_h_;
        // InitDevice of a CUDA build (cnn_detector_v3.cpp:73-84): packet mode forces the GPU pipeline
        if (cnn_ap_.packet_detection && cnn_p_.pipeline > 0 && cnn_ap_.detect_precision != CCNN_PRECISION_DEF) p->pipeline = CCNN_PIPELINE_GPU;
    }
    if (ap) {
        *ap = cnn_ap_;
        // the values CNNDetector::Init leaves in advanced_param (:922-963), and what Detect changed since
        // (apply_precision derives them again from the given values at every initialisation; the
        // gray-only state is Detect's, kept as it is)
        const bool gray_only = gray_image_only_;
        apply_precision();
        gray_image_only_ = gray_only;
        ap->type_check = type_check_;
        ap->min_num_detect = min_num_detect_;
        ap->drop_detect = drop_detect_;
        ap->equalize = equalize_;
        ap->reflection = reflection_;
        ap->adapt_min_neighbors = adapt_min_neighbors_;
        ap->double_check = double_check_;
        ap->merger_detect = merger_detect_;
        ap->gray_image_only = gray_image_only_;
        ap->facial_analysis = api_.facial_analysis;
        if (cnn_ap_.detect_precision == CCNN_PRECISION_DEF) {
            ap->packet_detection = 0;
            ap->blur = 0;
            ap->uniform_noise = 0;
        }
        if (cnn_p_.pipeline == CCNN_PIPELINE_CPU) ap->packet_detection = 0;  // InitDevice (:73-84)
    }
    return CCNN_OK;
}

ccnn_status Detector::set_cnn_params(const ccnn_cnn_param* p, const ccnn_cnn_advanced_param* ap) {
    std::lock_guard<std::mutex> lk(mu_);
    if (!has_cnn_) {
        set_error("the handle was not created through the CNNDetector API");
        return CCNN_ERR_INVALID_ARG;
    }
    if (ap) {
        const ccnn_status cs = check_cnn_params(*ap);
        if (cs != CCNN_OK) return cs;
    }
    clear();  // setParam / setAdvancedParam clear the detector (cnn_detector_v3.h:407-416)
    if (p) cnn_p_ = *p;
    if (ap) {
        cnn_ap_ = *ap;
        gray_image_only_ = ap->gray_image_only != 0;
    }
    cnn_to_api();
    max_w_ = cnn_p_.max_image_width;
    max_h_ = cnn_p_.max_image_height;
    return CCNN_OK;  // the next Detect initialises again (:2485-2492)
}

}  // namespace ccnn
