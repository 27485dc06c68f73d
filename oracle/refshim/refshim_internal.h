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
    int channels, elem_bytes, layers; /* images: channels per texel, bytes per channel, array layers */
    cl_channel_type channel_type;
};
struct UfoBuffer {
    UfoRequisition req;
    float *data;
    struct refshim_mem mem;
};
struct refshim_sampler {
    int bits; /* CLK_* sampler bits of the kernel-side shim */
};
#define REFSHIM_MAX_ARGS 128
struct refshim_kernel {
    char name[64];
    unsigned char args[REFSHIM_MAX_ARGS][64];
    size_t arg_size[REFSHIM_MAX_ARGS];
    struct refshim_jit *jit; /* kernels compiled at run time (ref_clc_jit.cpp) */
};
void refshim_buffer_init(struct UfoBuffer *b, float *data, guint n_dims, gsize d0, gsize d1, gsize d2);
void refshim_buffer_init_bytes(struct UfoBuffer *b, void *data, size_t bytes, guint n_dims, gsize d0, gsize d1,
                               gsize d2);
void refshim_dispatch(struct refshim_kernel *k, guint ndims, const gsize *global);
void refshim_jit_dispatch(struct refshim_kernel *k, guint ndims, const gsize *global, const gsize *local);
cl_kernel refshim_jit_from_file(const char *file, const char *name, GError **err);
void refshim_fft(float *data, size_t n, size_t batch, int forward);
/* Device limits reported by ufo_gpu_node_get_info (settable so that the
 * tasks' chunking paths can be exercised on small volumes). */
void refshim_set_device_limits(unsigned long global_mem, unsigned long max_alloc, unsigned long max_work_group);
/* Where ufo_resources_get_kernel_source finds the reference's kernel sources,
 * where the run-time kernel prelude lives, and where compiled kernels are cached. */
void refshim_set_dirs(const char *kernels_dir, const char *shim_dir, const char *cache_dir);
#ifdef __cplusplus
}
#endif
#endif
