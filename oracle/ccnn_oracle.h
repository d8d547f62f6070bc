/* Test infrastructure only — CPU restatement of the reference's detection path, used as the
 * checker by tests/, __graft_entry__.smoke() and bench.py's CPU baseline. Never part of the product.
 * Parity of this restatement with the reference is pinned by tests/golden (fixtures generated from
 * the reference's own code) and, where the reference build exists, by direct comparison. */
#ifndef CCNN_ORACLE_H
#define CCNN_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int max_image_w, max_image_h;
    int min_face_height, max_face_height;
    float scale_factor;
    int min_neighbors;
    int detect_precision;
    float treshold[3];
    int drop_detect, equalize, reflection;
    int detect_mode;
} orc_params;

typedef struct {
    int x, y, w, h;
    float score, scale;
    int knn, num_detect;
} orc_det;

typedef struct {
    int level, x, y;
    float score;
} orc_cand;

int orc_gray(const uint8_t* img, int w, int h, int ch, int step, float* out);
int orc_resize_f32(const float* src, int sw, int sh, int sstride, float* dst, int dw, int dh, int type);
int orc_equalize(uint8_t* img, int w, int h);
/* one network (model file) on one fp32 image; response map dense */
int orc_net_forward(const char* model_path, int index_output, const float* img, int w, int h, int stride, float* out, int cap, int* ow,
                    int* oh);
/* full detection with intermediates (see ccnn_oracle.cpp); returns the number of final boxes */
int orc_detect(const orc_params* p, const char* model_dir, const uint8_t* img, int w, int h, int ch, int step, float* gray_out,
               int* gray_w, int* gray_h, int level_cap, int* n_levels, float* scales, int* level_w, int* level_h, float* resp_out,
               long resp_cap, int* resp_w, int* resp_h, orc_cand* cands, int cand_cap, int* n_cands, orc_det* raw, int raw_cap,
               int* n_raw, orc_det* final_out, int final_cap);
/* std::sort permutation for comp(a, b) = b.scale < a.scale */
int orc_sort_perm(const float* keys, int n, int* perm);

#ifdef __cplusplus
}
#endif
#endif
