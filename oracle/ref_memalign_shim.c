/* Test infrastructure only. The reference's TmpImage asks posix_memalign for an alignment of
 * sizeof(uchar) == 1 (src/CNNObjectDetector/image.h:120), which glibc rejects (EINVAL, NULL
 * result, then a crash). image.cpp is compiled with -Dposix_memalign=ref_posix_memalign so its
 * one call lands here, where the alignment is raised to a valid power of two >= sizeof(void*). */
#include <stdlib.h>

int ref_posix_memalign(void** p, size_t align, size_t size) {
    size_t a = sizeof(void*);
    while (a < align) a <<= 1;
    return posix_memalign(p, a, size ? size : 1);
}
