// Serving loop: continuous batching of frames of mixed resolutions (include/ccnn_server.h).
//
// One scheduler thread owns every CUDA call of the server. Callers only touch the request queue
// and the finished results, under one mutex. The scheduler repeatedly
//   1. collects finished slots (event queries, no blocking), hands their faces to the requests and
//      wakes the waiters;
//   2. admits queued requests in arrival order onto free slots of their resolution class,
//      creating the class (a Detector sized for exactly that frame) when the HBM budget allows,
//      after evicting idle classes, least recently used first.
// Each slot runs the captured per-frame graph of the plain cascade on its own stream, so frames
// of different classes and different slots overlap on the device.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <memory>
#include <thread>
#include <vector>
#include <unordered_map>

#include "../../include/ccnn_server.h"
#include "detector.h"

extern "C" const char* ccnn_last_error(void);

namespace ccnn {

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kResultCap = Detector::kHostFaces;

struct Request {
    long long ticket = 0;
    ccnn_image img{};
    Clock::time_point t_submit, t_done;
    std::vector<ccnn_face> faces;
    int n = 0;
    ccnn_status status = CCNN_PENDING;
    std::string error;
};

struct ResClass {
    int w = 0, h = 0, c = 0;
    std::unique_ptr<Detector> det;
    std::vector<std::shared_ptr<Request>> slot_req;  // request on each slot, null when free
    int busy = 0;
    long long last_used = 0;
    size_t bytes = 0;
    bool match(const ccnn_image& im) const { return im.cols == w && im.rows == h && im.channels == c; }
};

}  // namespace

class Server {
   public:
    ccnn_status create(const ccnn_params& p, const char* const* models, const ccnn_server_config* cfg);
    ~Server();
    ccnn_status submit(const ccnn_image& img, long long* ticket);
    ccnn_status set_gate(const float* params, int n, float threshold, float fallback_fraction);
    ccnn_status set_gate_margin(int pixels);
    ccnn_status take(long long ticket, bool block, ccnn_face* faces, int cap, int* n, double* lat);
    void stats(ccnn_server_stats* out);

   private:
    void loop();
    bool collect_finished();
    bool admit();
    ResClass* find_class(const ccnn_image& img);
    ccnn_status make_class(const ccnn_image& img, ResClass** out, bool* retry_later);
    void fail(const std::shared_ptr<Request>& r, ccnn_status st, const std::string& why);

    ccnn_params params_{};
    std::vector<float> gate_;  // learned-gate parameters for every class (empty: full scan)
    std::vector<ccnn_face> fetch_buf_;  // results of a finished slot (scheduler thread only)
    float gate_thr_ = 0.5f, gate_fb_ = 0.25f;
    int gate_margin_ = 16;
    std::string models_[3];
    bool has_models_ = false;
    size_t budget_ = 0;
    int slots_per_class_ = 4;
    int max_queue_ = 65536;

    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    std::deque<std::shared_ptr<Request>> queue_;
    std::unordered_map<long long, std::shared_ptr<Request>> open_;  // results not taken yet
    long long next_ticket_ = 1;
    long long submitted_ = 0, completed_ = 0, failed_ = 0;
    int in_flight_ = 0;
    std::atomic<bool> stop_{false};

    // scheduler-thread state
    std::list<std::unique_ptr<ResClass>> classes_;
    std::atomic<size_t> held_{0};   // read by stats() on caller threads
    std::atomic<int> n_classes_{0};
    long long clock_ = 0;
    bool blocked_on_budget_ = false;  // a class creation failed for room: retry after a completion
    std::thread thread_;
};

ccnn_status Server::create(const ccnn_params& p, const char* const* models, const ccnn_server_config* cfg) {
    params_ = p;
    if (models) {
        has_models_ = true;
        for (int i = 0; i < 3; ++i) models_[i] = models[i] ? models[i] : "";
    }
    budget_ = (cfg && cfg->hbm_budget_bytes) ? cfg->hbm_budget_bytes : (size_t)8 << 30;
    slots_per_class_ = (cfg && cfg->slots_per_class > 0) ? cfg->slots_per_class : 4;
    max_queue_ = (cfg && cfg->max_queue > 0) ? cfg->max_queue : 65536;
    // validate the parameters and models once, on the caller's thread
    Detector probe;
    ccnn_params pp = p;
    const char* mp[3] = {models_[0].c_str(), models_[1].c_str(), models_[2].c_str()};
    ccnn_status st = probe.create(pp, has_models_ ? mp : nullptr, 1, false);
    if (st != CCNN_OK) return st;
    thread_ = std::thread(&Server::loop, this);
    return CCNN_OK;
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_.store(true);
    }
    cv_work_.notify_all();
    if (thread_.joinable()) thread_.join();
}

// The gate is fixed before the first frame: every class is then created with it.
ccnn_status Server::set_gate(const float* params, int n, float threshold, float fallback_fraction) {
    if (!params || n != kGateParams || !(threshold > 0.f && threshold < 1.f) || !(fallback_fraction >= 0.f)) {
        set_error("gate: kGateParams parameters, a threshold in (0, 1) and a non-negative fallback fraction are needed");
        return CCNN_ERR_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lk(mu_);
    if (submitted_ > 0) {
        set_error("the gate must be set before the first frame is submitted");
        return CCNN_ERR_INVALID_ARG;
    }
    gate_.assign(params, params + n);
    gate_thr_ = threshold;
    gate_fb_ = fallback_fraction;
    return CCNN_OK;
}

ccnn_status Server::set_gate_margin(int pixels) {
    if (pixels < 0 || pixels > 64) {
        set_error("gate margin: 0-64 pixels");
        return CCNN_ERR_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lk(mu_);
    if (submitted_ > 0) {
        set_error("the gate margin must be set before the first frame is submitted");
        return CCNN_ERR_INVALID_ARG;
    }
    gate_margin_ = pixels;
    return CCNN_OK;
}

ccnn_status Server::submit(const ccnn_image& img, long long* ticket) {
    if (!ticket || img.cols <= 0 || img.rows <= 0 || !img.data || img.step < (size_t)img.cols * img.channels) {
        set_error("invalid image");
        return CCNN_ERR_INVALID_ARG;
    }
    if (img.channels != 1 && img.channels != 3 && img.channels != 4) {
        set_error("this type of image is not supported (1, 3 or 4 channels)");
        return CCNN_ERR_UNSUPPORTED;
    }
    auto r = std::make_shared<Request>();
    r->img = img;
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(mu_);
        if ((int)queue_.size() >= max_queue_) return CCNN_BUSY;
        r->ticket = next_ticket_++;
        queue_.push_back(r);
        open_[r->ticket] = r;
        submitted_++;
        *ticket = r->ticket;
    }
    cv_work_.notify_one();
    return CCNN_OK;
}

ccnn_status Server::take(long long ticket, bool block, ccnn_face* faces, int cap, int* n, double* lat) {
    if (!n || cap < 0 || (cap > 0 && !faces)) {
        set_error("invalid output arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    std::unique_lock<std::mutex> lk(mu_);
    auto it = open_.find(ticket);
    if (it == open_.end()) {
        set_error("unknown ticket (never submitted, or its result was already taken)");
        return CCNN_ERR_INVALID_ARG;
    }
    std::shared_ptr<Request> r = it->second;
    if (r->status == CCNN_PENDING) {
        if (!block) return CCNN_PENDING;
        cv_done_.wait(lk, [&] { return r->status != CCNN_PENDING; });
    }
    open_.erase(ticket);
    lk.unlock();
    if (lat) *lat = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    if (r->status < 0) {
        set_error(r->error);
        *n = 0;
        return r->status;
    }
    *n = r->n;
    const int take = std::min(std::min(r->n, cap), (int)r->faces.size());
    for (int i = 0; i < take; ++i) faces[i] = r->faces[i];
    return r->n > cap ? CCNN_TRUNCATED : r->status;
}

void Server::stats(ccnn_server_stats* out) {
    std::lock_guard<std::mutex> lk(mu_);
    out->submitted = submitted_;
    out->completed = completed_;
    out->failed = failed_;
    out->queued = (int)queue_.size();
    out->in_flight = in_flight_;
    out->classes = n_classes_.load();
    out->hbm_bytes = held_.load();
}

void Server::fail(const std::shared_ptr<Request>& r, ccnn_status st, const std::string& why) {
    std::lock_guard<std::mutex> lk(mu_);
    r->status = st;
    r->error = why;
    r->t_done = Clock::now();
    failed_++;
    cv_done_.notify_all();
}

ResClass* Server::find_class(const ccnn_image& img) {
    for (auto& c : classes_)
        if (c->match(img)) return c.get();
    return nullptr;
}

// A detector for exactly this frame size: the result of every frame then equals ccnn_detect on
// a fresh handle whose max_image_size is the frame (no re-initialisation, no level-count state).
ccnn_status Server::make_class(const ccnn_image& img, ResClass** out, bool* retry_later) {
    *retry_later = false;
    ccnn_params p = params_;
    p.max_image_width = img.cols;
    p.max_image_height = img.rows;
    const char* mp[3] = {models_[0].c_str(), models_[1].c_str(), models_[2].c_str()};
    const char* const* models = has_models_ ? mp : nullptr;
    const bool colour = img.channels != 1;
    // evicts the least recently used idle class; false when every class is busy
    auto evict_one = [&]() {
        ResClass* victim = nullptr;
        for (auto& o : classes_)
            if (o->busy == 0 && (!victim || o->last_used < victim->last_used)) victim = o.get();
        if (!victim) return false;
        held_ -= victim->bytes;
        classes_.remove_if([&](const std::unique_ptr<ResClass>& o) { return o.get() == victim; });
        n_classes_ = (int)classes_.size();
        return true;
    };
    for (int slots = slots_per_class_; slots >= 1; slots /= 2) {
        // the class's device bytes are known from its plan before anything is allocated, so room
        // is made first (idle classes evicted, least recently used first) and the budget is never
        // exceeded, not even briefly
        size_t bytes = 0;
        ccnn_status st = Detector::estimate_bytes(p, models, slots, colour, !gate_.empty(), &bytes);
        if (st != CCNN_OK) return st;
        while (held_ + bytes > budget_ && evict_one()) {
        }
        if (held_ + bytes > budget_) {
            bool busy = false;
            for (auto& o : classes_) busy |= o->busy > 0;
            if (busy) {  // room comes back when running frames finish
                *retry_later = true;
                return CCNN_OK;
            }
            continue;  // fewer slots
        }
        std::unique_ptr<ResClass> c(new ResClass());
        c->w = img.cols;
        c->h = img.rows;
        c->c = img.channels;
        // the device itself may hold less than the budget: on OOM, evict another idle class and retry
        for (;;) {
            c->det.reset(new Detector());
            st = c->det->create(p, models, slots, colour);
            if (st == CCNN_OK && !gate_.empty()) st = c->det->gate_set(gate_.data(), (int)gate_.size(), gate_thr_, gate_fb_);
            if (st == CCNN_OK && !gate_.empty()) st = c->det->gate_set_margin(gate_margin_);
            if (st != CCNN_ERR_OOM || !evict_one()) break;
        }
        if (st == CCNN_ERR_OOM) {
            c->det.reset();
            bool busy = false;
            for (auto& o : classes_) busy |= o->busy > 0;
            if (busy) {
                *retry_later = true;
                return CCNN_OK;
            }
            continue;  // fewer slots
        }
        if (st != CCNN_OK) return st;
        c->bytes = c->det->slot_bytes();
        c->slot_req.assign(slots, nullptr);
        held_ += c->bytes;
        classes_.push_back(std::move(c));
        n_classes_ = (int)classes_.size();
        *out = classes_.back().get();
        return CCNN_OK;
    }
    set_error("a frame of this size does not fit the server's HBM budget");
    return CCNN_ERR_OOM;
}

bool Server::collect_finished() {
    bool progress = false;
    for (auto& c : classes_) {
        for (int k = 0; k < (int)c->slot_req.size(); ++k) {
            std::shared_ptr<Request>& r = c->slot_req[k];
            if (!r || !c->det->slot_done(k)) continue;
            // fetched into one reusable buffer; the request keeps only its own faces
            if (fetch_buf_.size() < (size_t)kResultCap) fetch_buf_.resize(kResultCap);
            int n = 0;
            const ccnn_status st = c->det->fetch(k, fetch_buf_.data(), kResultCap, &n);
            const std::string err = st < 0 ? std::string(ccnn_last_error()) : std::string();
            std::vector<ccnn_face> faces(fetch_buf_.begin(), fetch_buf_.begin() + (st < 0 ? 0 : std::min(std::max(n, 0), kResultCap)));
            {
                std::lock_guard<std::mutex> lk(mu_);
                r->faces.swap(faces);
                r->n = n;
                r->status = st < 0 ? st : CCNN_OK;
                r->error = err;
                r->t_done = Clock::now();
                if (st < 0) failed_++;
                else completed_++;
                in_flight_--;
            }
            cv_done_.notify_all();
            r.reset();
            c->busy--;
            blocked_on_budget_ = false;
            progress = true;
        }
    }
    return progress;
}

bool Server::admit() {
    bool progress = false;
    while (true) {
        std::shared_ptr<Request> r;
        ResClass* cls = nullptr;
        int slot = -1;
        bool need_class = false;
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (auto it = queue_.begin(); it != queue_.end(); ++it) {
                ResClass* c = find_class((*it)->img);
                if (!c) {
                    if (blocked_on_budget_) continue;
                    r = *it;
                    need_class = true;
                    break;
                }
                int k = -1;
                for (int q = 0; q < (int)c->slot_req.size(); ++q)
                    if (!c->slot_req[q]) {
                        k = q;
                        break;
                    }
                if (k < 0) continue;  // this class is full; later requests of other classes may run
                r = *it;
                cls = c;
                slot = k;
                queue_.erase(it);
                in_flight_++;
                break;
            }
        }
        if (!r) return progress;
        if (need_class) {
            bool retry = false;
            ResClass* c = nullptr;
            const ccnn_status st = make_class(r->img, &c, &retry);
            if (st != CCNN_OK) {
                {
                    std::lock_guard<std::mutex> lk(mu_);
                    for (auto it = queue_.begin(); it != queue_.end(); ++it)
                        if (*it == r) {
                            queue_.erase(it);
                            break;
                        }
                }
                fail(r, st, ccnn_last_error());
            } else if (retry) {
                blocked_on_budget_ = true;
            }
            progress = true;
            continue;
        }
        cls->slot_req[slot] = r;
        cls->busy++;
        cls->last_used = ++clock_;
        const ccnn_status st = cls->det->launch(slot, r->img);
        if (st != CCNN_OK) {
            cls->slot_req[slot].reset();
            cls->busy--;
            {
                std::lock_guard<std::mutex> lk(mu_);
                in_flight_--;
            }
            fail(r, st, ccnn_last_error());
        }
        progress = true;
    }
}

void Server::loop() {
    while (true) {
        {
            std::unique_lock<std::mutex> lk(mu_);
            if (stop_ && in_flight_ == 0) break;
            if (queue_.empty() && in_flight_ == 0) {
                cv_work_.wait(lk, [&] { return stop_ || !queue_.empty(); });
                continue;
            }
        }
        const bool a = collect_finished();
        const bool b = stop_.load() ? false : admit();
        if (!a && !b) std::this_thread::sleep_for(std::chrono::microseconds(5));
    }
    // requests still queued at shutdown
    std::lock_guard<std::mutex> lk(mu_);
    for (auto& r : queue_) {
        r->status = CCNN_ERR_INVALID_ARG;
        r->error = "server destroyed before the frame ran";
        r->t_done = Clock::now();
    }
    queue_.clear();
    cv_done_.notify_all();
}

}  // namespace ccnn

struct ccnn_server_s {
    ccnn::Server srv;
};

extern "C" CCNN_API ccnn_status ccnn_server_create(const ccnn_params* params, const char* const* model_paths,
                                                   const ccnn_server_config* config, ccnn_server* out) {
    if (!params || !out) {
        ccnn::set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    std::unique_ptr<ccnn_server_s> s(new ccnn_server_s());
    const ccnn_status st = s->srv.create(*params, model_paths, config);
    if (st != CCNN_OK) return st;
    *out = s.release();
    return CCNN_OK;
}

extern "C" CCNN_API ccnn_status ccnn_server_set_gate_margin(ccnn_server s, int pixels) {
    if (!s) {
        ccnn::set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    return s->srv.set_gate_margin(pixels);
}

extern "C" CCNN_API ccnn_status ccnn_server_set_gate(ccnn_server s, const float* params, int n_params, float threshold,
                                                     float fallback_fraction) {
    if (!s) {
        ccnn::set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    return s->srv.set_gate(params, n_params, threshold, fallback_fraction);
}

extern "C" CCNN_API ccnn_status ccnn_server_destroy(ccnn_server s) {
    delete s;
    return CCNN_OK;
}

extern "C" CCNN_API ccnn_status ccnn_server_submit(ccnn_server s, const ccnn_image* img, long long* ticket) {
    if (!s || !img) {
        ccnn::set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    return s->srv.submit(*img, ticket);
}

extern "C" CCNN_API ccnn_status ccnn_server_poll(ccnn_server s, long long ticket, ccnn_face* faces, int capacity, int* n_faces,
                                                 double* latency_ms) {
    if (!s) {
        ccnn::set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    return s->srv.take(ticket, false, faces, capacity, n_faces, latency_ms);
}

extern "C" CCNN_API ccnn_status ccnn_server_wait(ccnn_server s, long long ticket, ccnn_face* faces, int capacity, int* n_faces,
                                                 double* latency_ms) {
    if (!s) {
        ccnn::set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    return s->srv.take(ticket, true, faces, capacity, n_faces, latency_ms);
}

extern "C" CCNN_API ccnn_status ccnn_server_stats_get(ccnn_server s, ccnn_server_stats* out) {
    if (!s || !out) {
        ccnn::set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    s->srv.stats(out);
    return CCNN_OK;
}

extern "C" CCNN_API void* ccnn_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    return p;
}

extern "C" CCNN_API void ccnn_host_free(void* p) {
    if (p) cudaFreeHost(p);
}
