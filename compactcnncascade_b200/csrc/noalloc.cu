// Stage-1 net on one device image with no device allocation at all.
//
// Who needs this: callers that are not allowed to call cudaMalloc — plug-in hosts that account for
// every byte of device memory up front and hand a component only its input and output buffers, or
// processes whose device memory is already fully reserved by another framework's caching
// allocator, where an extra cudaMalloc would fail (or stall the device while memory is freed).
// The regular entry points allocate per-handle buffers; this one uses a fixed scratch array that is
// part of the library image instead.
//
// The scratch is a file-scope __device__ array: every GPU that loads the library holds it (9 MiB +
// 256 B) until the process exits. It holds the four L1 neighbour-sum planes of the image (up to
// kStaticS1Floats floats) after a reserved first 256 bytes; the level descriptor travels as a
// kernel parameter. Every call shares it, and it keeps the last call's contents; nothing in it has
// to start at zero, because each call writes every plane value it later reads. Calls that overlap
// on the GPU (different streams, or different host threads) race on the array. The array's device
// address is looked up once per CUDA context, so a device reset between calls is handled (the next
// call looks it up again in the new context).
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>

#include "../../include/ccnn_inspect.h"
#include "kernels.h"
#include "model.h"

namespace ccnn {

void set_error(const std::string& msg);

namespace {

constexpr long long kStaticS1Floats = 2359296;  // 9 MiB of fp32: a 1920x1080 image needs 2,065,920
constexpr size_t kDescBytes = 256;  // reserved head of the array

static __device__ __align__(256) unsigned char g_stage1_scratch[kDescBytes + sizeof(float) * kStaticS1Floats];

std::mutex g_mu;
std::map<unsigned long long, void*> g_scratch_addr;  // per CUDA context: the array's device address
std::map<std::string, Stage1W> g_weights;

// Identity of the calling thread's current CUDA context. A device reset (cudaDeviceReset) ends the
// context and reloads the library's module into the next one, which moves the array and drops the
// kernel attributes, so both are cached per context rather than per device ordinal. The driver's
// cuCtxGetCurrent / cuCtxGetId are reached through the runtime's entry-point query, so the library
// does not link libcuda itself.
ccnn_status current_context_id(unsigned long long* id) {
    typedef int (*GetCurrentFn)(void**);
    typedef int (*GetIdFn)(void*, unsigned long long*);
    static GetCurrentFn get_current = nullptr;
    static GetIdFn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        cudaDriverEntryPointQueryResult q1, q2;
        void* f1 = nullptr;
        void* f2 = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrentFn>(f1);
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) == cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetIdFn>(f2);
        looked_up = true;
    }
    void* ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, id) != 0) {
        set_error("static stage-1 scratch: cannot identify the current CUDA context (driver entry points cuCtxGetCurrent/cuCtxGetId)");
        return CCNN_ERR_CUDA;
    }
    return CCNN_OK;
}

// One-time set-up per CUDA context (the calling thread's device current): the device address of
// the array and the stage-1 kernel attribute. Neither allocates.
ccnn_status scratch_address(unsigned char** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    unsigned long long ctx = 0;
    const ccnn_status cs = current_context_id(&ctx);
    if (cs != CCNN_OK) return cs;
    auto it = g_scratch_addr.find(ctx);
    if (it == g_scratch_addr.end()) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_stage1_scratch);
        if (e != cudaSuccess) {
            set_error(std::string("cudaGetSymbolAddress(static stage-1 scratch): ") + cudaGetErrorString(e));
            return CCNN_ERR_CUDA;
        }
        const cudaError_t e2 = stage1_setup();  // kernel attribute, no allocation
        if (e2 != cudaSuccess) {
            set_error(std::string("stage-1 kernel set-up: ") + cudaGetErrorString(e2));
            return CCNN_ERR_CUDA;
        }
        it = g_scratch_addr.emplace(ctx, p).first;
    }
    *out = static_cast<unsigned char*>(it->second);
    return CCNN_OK;
}

ccnn_status stage1_weights(const char* model_path, Stage1W* w) {
    const std::string path = (model_path && model_path[0]) ? std::string(model_path) : bundled_model_dir() + "/cnn4face1_cntk.bin";
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_weights.find(path);
    if (it == g_weights.end()) {
        RawModel m;
        std::string err;
        Stage1W packed;
        if (!load_model_file(path, &m, &err) || !pack_model(m, 1, &packed, &err)) {
            set_error(err);
            return CCNN_ERR_MODEL;
        }
        if (m.min_w != kPatW || m.min_h != kPatH) {
            set_error("stage-1 model window is not 23x27");
            return CCNN_ERR_MODEL;
        }
        it = g_weights.emplace(path, packed).first;
    }
    *w = it->second;
    return CCNN_OK;
}

}  // namespace
}  // namespace ccnn

extern "C" CCNN_API ccnn_status ccnn_stage1_forward_static(const char* model_path, const float* d_img, int cols, int rows, size_t step,
                                                           float* d_resp, int resp_cap, int* resp_cols, int* resp_rows, void* stream) {
    using namespace ccnn;
    if (!d_img || !d_resp || !resp_cols || !resp_rows || (step % sizeof(float)) != 0 || step < sizeof(float) * (size_t)cols) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    if (cols < kPatW || rows < kPatH) {
        set_error("image smaller than the 23x27 stage-1 window");
        return CCNN_ERR_INVALID_ARG;
    }
    LevelDesc L{};
    L.w = cols;
    L.h = rows;
    L.mode = 0;
    L.scale = 1.f;
    L.inv_scale = 1.f;
    L.p1w = (cols - 3) >> 1;
    L.p1h = (rows - 3) >> 1;
    L.p2w = (L.p1w - 2) >> 1;
    L.p2h = (L.p1h - 2) >> 1;
    L.ow = L.p2w - 3;
    L.oh = L.p2h - 4;
    L.s1_pitch = (L.p1w + 31) / 32 * 32;
    L.s1_plane = (long long)L.s1_pitch * L.p1h;
    L.s1_off = 0;
    L.resp_off = 0;
    L.k1_tiles_x = (L.p1w + kK1TileX - 1) / kK1TileX;
    L.k2_tiles_x = (L.ow + kK2TileX - 1) / kK2TileX;
    L.k1_base = 0;
    L.k2_base = 0;
    L.img_off = 0;
    L.img_pitch = (int)(step / sizeof(float));
    L.img_vec = (L.img_pitch % 4 == 0 && (reinterpret_cast<uintptr_t>(d_img) & 15) == 0) ? 1 : 0;
    *resp_cols = L.ow;
    *resp_rows = L.oh;
    if (4 * L.s1_plane > kStaticS1Floats) {
        set_error("image too large for the static scratch: its four L1 planes need " + std::to_string(4 * L.s1_plane) +
                  " floats, the maximum is 2359296 (about 1920x1080 or 2^21 pixels)");
        return CCNN_ERR_INVALID_ARG;
    }
    if ((long long)L.ow * L.oh > resp_cap) {
        set_error("response capacity too small");
        return CCNN_ERR_INVALID_ARG;
    }
    Stage1W w;
    ccnn_status st = stage1_weights(model_path, &w);
    if (st != CCNN_OK) return st;
    // cudaSetDevice on the current device makes sure its primary context exists and is current
    // before the context is identified (it allocates nothing)
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaSetDevice(dev);
    if (e != cudaSuccess) {
        set_error(std::string("cudaGetDevice/cudaSetDevice: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    unsigned char* scratch = nullptr;
    st = scratch_address(&scratch);
    if (st != CCNN_OK) return st;
    float* d_s1 = reinterpret_cast<float*>(scratch + kDescBytes);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    e = launch_stage1_front(w, &L, 1, d_img, d_s1, s);
    if (e == cudaSuccess) e = launch_stage1_back(w, &L, 1, d_s1, d_resp, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(std::string("static stage-1 forward: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    return CCNN_OK;
}
