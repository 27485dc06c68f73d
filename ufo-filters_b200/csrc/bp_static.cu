// Allocation-free parallel-beam backprojection.
//
// ufob_backproject_run() keeps its per-angle sin/cos table in device memory
// that the handle allocates on first use (and restages sinograms whose rows are
// not 16-byte aligned into another allocated buffer).  Some callers cannot call
// cudaMalloc at all: hosts that own every byte of device memory through their
// own pool and forbid outside allocations, and acquisition pipelines that must
// not take the device-wide synchronisation an allocation can imply while frames
// are streaming.  For them this file provides
// ufob_backproject_run_static(): the same kernels, with the only scratch they
// need -- the angle table -- in a fixed file-scope device array.  The result
// equals ufob_backproject_run()'s within round-off: a single sinogram is not
// split into angle groups here.
//
// Limits and sharing rules (also stated in ufob.h):
//  * at most UFOB_STATIC_MAX_ANGLES sinogram rows per call;
//  * rows must already be 16-byte aligned (TMA); nothing is restaged;
//  * the array is shared by every call in the process and keeps the last
//    call's table; each call rewrites the entries it uses before its kernel
//    reads them, so nothing has to start at zero, but calls whose work overlaps
//    on the GPU (different streams, no ordering) race on the table;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (device set-up); make that first call before any
//    stream capture.
#include <math.h>

#include <atomic>

#include "ufob_internal.h"

namespace ufob {

// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) float2 g_static_sincos[UFOB_STATIC_MAX_ANGLES];

static constexpr int kMaxDevices = 64;
// device address of g_static_sincos per device; host threads that make their
// first call at the same time both look it up and store the same value
static std::atomic<float2 *> g_static_ptr[kMaxDevices];

// Per-device set-up: host code may not pass the array's name to a kernel (on
// the host it is only a stand-in symbol), so look its device address up once
// per device, with that device current.
static ufob_status static_table_address(float2 **out)
{
    int dev = 0;
    UFOB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(UFOB_ERR_UNSUPPORTED, "device index %d out of range", dev);
    float2 *ptr = g_static_ptr[dev].load(std::memory_order_acquire);
    if (!ptr) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_sincos);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static angle table)");
        ptr = reinterpret_cast<float2 *>(p);
        g_static_ptr[dev].store(ptr, std::memory_order_release);
    }
    *out = ptr;
    return UFOB_OK;
}

}  // namespace ufob

using namespace ufob;

extern "C" ufob_status ufob_backproject_run_static(const ufob_bp_props *props, const void *d_sino,
                                                   ufob_dtype dtype, ufob_layout layout, uint32_t width,
                                                   uint32_t height, uint32_t nslices, uint32_t pitch,
                                                   uint64_t slice_pitch, float *d_out, void *stream)
{
    if (!props || !d_sino || !d_out) return fail(UFOB_ERR_INVALID, "backproject_run_static: NULL argument");
    const ufob_bp_props &p = *props;
    if (p.num_projections > 32768 || p.offset > 32768 || !(p.axis_pos >= -1.0 && p.axis_pos <= 32768.0) ||
        !(p.angle_offset >= 0.0) || (p.mode != UFOB_BP_NEAREST && p.mode != UFOB_BP_TEXTURE))
        return fail(UFOB_ERR_INVALID, "backproject_run_static: property out of range");
    if (!width || !height) return fail(UFOB_ERR_REQUISITION, "backproject: empty sinogram %ux%u", width, height);
    if (height > UFOB_STATIC_MAX_ANGLES)
        return fail(UFOB_ERR_UNSUPPORTED,
                    "backproject_run_static: %u sinogram rows exceed the static angle table (%u rows); "
                    "use ufob_backproject_run",
                    height, (unsigned)UFOB_STATIC_MAX_ANGLES);
    // requisition rules of src/ufo-backproject-task.c:212-267
    const uint32_t nproj = p.num_projections ? p.num_projections : height;
    if (height > nproj)
        return fail(UFOB_ERR_REQUISITION,
                    "Total number of projections (%u) must be greater than or equal to sinogram height (%u)", nproj,
                    height);
    if ((uint64_t)p.offset + height > nproj)
        return fail(UFOB_ERR_REQUISITION, "offset (%u) + sinogram height (%u) exceeds the %u angle table entries",
                    p.offset, height, nproj);
    SinoKind kind;
    if (dtype == UFOB_F32 && layout == UFOB_LAYOUT_ROWS) kind = SINO_F32;
    else if (dtype == UFOB_F16 && layout == UFOB_LAYOUT_PAIRS) kind = SINO_F16_PAIRS;
    else if (dtype == UFOB_BF16 && layout == UFOB_LAYOUT_PAIRS) kind = SINO_BF16_PAIRS;
    else return fail(UFOB_ERR_INVALID, "backproject: sinogram must be F32 rows or F16/BF16 pairs");
    const uint32_t elems = kind == SINO_F32 ? width : width + 1;
    if (!pitch) pitch = kind == SINO_F32 ? width : round_up(width + 1, 4);
    if (pitch < elems) return fail(UFOB_ERR_INVALID, "backproject: pitch %u < row length %u", pitch, elems);
    if (!slice_pitch) slice_pitch = (uint64_t)pitch * height;
    if (p.mode != UFOB_BP_NEAREST && (((uintptr_t)d_sino & 15) || (pitch & 3) || (slice_pitch & 3)))
        return fail(UFOB_ERR_INVALID,
                    "backproject_run_static: rows must be 16-byte aligned (base, pitch and slice pitch multiples of "
                    "4 elements); use ufob_backproject_run, which restages them");
    UFOB_TRY(ensure_device());
    float2 *table = nullptr;
    UFOB_TRY(static_table_address(&table));
    cudaStream_t s = (cudaStream_t)stream;
    const double step = p.angle_step > 0.0 ? p.angle_step : M_PI / (double)nproj;
    UFOB_TRY(sincos_table_launch(p.angle_offset, step, p.offset, height, table, s));
    BPGeometry g;
    g.W = width;
    g.P = height;
    g.nz = nslices;
    g.roi_x = p.roi_x;
    g.roi_y = p.roi_y;
    g.roi_w = p.roi_width ? p.roi_width : width;
    g.roi_h = p.roi_height ? p.roi_height : width;
    g.axis = p.axis_pos <= 0.0 ? (float)width / 2.0f : (float)p.axis_pos;
    g.norm = (float)M_PI / (float)height;
    g.d_sincos = table;
    if (p.mode == UFOB_BP_NEAREST) {
        if (kind != SINO_F32) return fail(UFOB_ERR_INVALID, "backproject: mode=nearest needs an F32 sinogram");
        return bp_nearest_launch(g, (const float *)d_sino, pitch, slice_pitch, d_out, s);
    }
    const bool kahan = p.compensated >= 0 ? p.compensated != 0 : (kind != SINO_F32 && height >= 1500);
    return bp_linear_launch(g, d_sino, kind, pitch, slice_pitch, d_out, kahan, p.tile, s);
}
