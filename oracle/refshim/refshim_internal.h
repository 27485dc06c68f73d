/* Shared definitions of the CPU runtime behind the reference shims. */
#ifndef REFSHIM_INTERNAL_H
#define REFSHIM_INTERNAL_H
#include <ufo/ufo.h>
#ifdef __cplusplus
extern "C" {
#endif
struct refshim_mem {
    size_t size;
    void *host;
    int is_image, width, height, owned;
};
struct UfoBuffer {
    UfoRequisition req;
    float *data;
    struct refshim_mem mem;
};
#define REFSHIM_MAX_ARGS 48
struct refshim_kernel {
    char name[64];
    unsigned char args[REFSHIM_MAX_ARGS][64];
    size_t arg_size[REFSHIM_MAX_ARGS];
};
void refshim_buffer_init(struct UfoBuffer *b, float *data, guint n_dims, gsize d0, gsize d1, gsize d2);
void refshim_dispatch(struct refshim_kernel *k, guint ndims, const gsize *global);
void refshim_fft(float *data, size_t n, size_t batch, int forward);
#ifdef __cplusplus
}
#endif
#endif
