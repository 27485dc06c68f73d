// Uneven batches of parallel-beam reconstructions (many independent
// `fft ! filter ! ifft ! backproject` graphs, as ufo-core runs one task
// instance per item) in one graph launch:
//   1. FP64 sin/cos tables of every job (one kernel, grid.y = job);
//   2. the filter stage of every job as one persistent kernel over
//      (job, row pair) items grouped by FFT width;
//   3. the backprojection of every job as one persistent kernel over
//      (job, tile) items ordered by decreasing angle count (largest first),
//      taken dynamically from a device counter.
// The three launches and the counter resets are captured into a CUDA graph on
// the first run of a batch and replayed while the batch (pointers, sizes,
// geometry) stays the same.  The tile shape of stage 3 is chosen by an
// autotuner that times every variant on the batch once and caches the winner
// on disk keyed by the batch's shape (UFOB_TUNE_CACHE, default
// $HOME/.cache/ufob/tune.txt; UFOB_TUNE=0 disables tuning).
//
// Per job the graph is `fft size-x=N ! filter ! ifft crop-width=W ! backproject`
// with N = fft size-x if set, else the next power of two >= W (the reference's
// filter needs a power-of-two spectrum width, src/ufo-filter-task.c:295-300),
// axis-pos W/2 unless given, angle-step pi/height unless given.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "ufob_internal.h"

namespace ufob {

__global__ void k_batch_sincos(const double *__restrict__ geo, const uint32_t *__restrict__ rows,
                               float2 *const *__restrict__ outs)
{
    const uint32_t j = blockIdx.y, p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= rows[j]) return;
    double s, c;
    sincos(geo[2 * j] + (double)p * geo[2 * j + 1], &s, &c);
    outs[j][p] = make_float2((float)s, (float)c);
}

static uint32_t next_pow2(uint32_t v)
{
    uint32_t n = 1;
    while (n < v) n <<= 1;
    return n;
}

static std::string tune_path()
{
    const char *p = getenv("UFOB_TUNE_CACHE");
    if (p && *p) return p;
    const char *home = getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/ufob/tune.txt";
}

static bool tune_lookup(const std::string &key, int *variant)
{
    FILE *f = fopen(tune_path().c_str(), "r");
    if (!f) return false;
    char k[512];
    int v;
    bool found = false;
    while (fscanf(f, "%511s %d", k, &v) == 2)
        if (key == k) {
            *variant = v;
            found = true;
        }
    fclose(f);
    return found;
}

static void tune_store(const std::string &key, int variant)
{
    std::string path = tune_path();
    std::string dir = path.substr(0, path.find_last_of('/'));
    std::string cmd = "mkdir -p '" + dir + "' 2>/dev/null";
    if (system(cmd.c_str()) != 0) return;
    FILE *f = fopen(path.c_str(), "a");
    if (!f) return;
    fprintf(f, "%s %d\n", key.c_str(), variant);
    fclose(f);
}

}  // namespace ufob

using namespace ufob;

struct ufob_batch {
    ufob_filter_props props;
    ufob_dtype storage;
    std::map<uint32_t, FilterPlan> plans;  // per FFT width
    DevBuf work, tables, d_fjobs, d_bjobs, d_fitems, d_bitems, d_counters, d_geo, d_rows, d_outs;
    // host copies (the device arrays are re-uploaded only when the batch changes)
    std::vector<BatchFilter> fjobs;
    std::vector<BatchBP> bjobs;
    std::vector<uint2> fitems, bitems;
    std::vector<double> geo;
    std::vector<uint32_t> rows;
    std::vector<float2 *> outs;
    std::string signature;
    int variant = -1;
    int pinned = -1;  // tile variant fixed by ufob_batch_set_variant, -1 = autotuned
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t maxN = 0, maxP = 0;
    ~ufob_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

extern "C" ufob_status ufob_batch_create(const ufob_filter_props *fprops, ufob_dtype storage, ufob_batch **out)
{
    if (!out) return fail(UFOB_ERR_INVALID, "batch_create: out is NULL");
    if (storage != UFOB_F32 && storage != UFOB_F16 && storage != UFOB_BF16)
        return fail(UFOB_ERR_INVALID, "batch: storage must be F32, F16 or BF16");
    ufob_batch *b = new ufob_batch;
    ufob_filter_props_init(&b->props);
    if (fprops) b->props = *fprops;
    b->storage = storage;
    *out = b;
    return UFOB_OK;
}

extern "C" void ufob_batch_destroy(ufob_batch *b) { delete b; }

// Enqueue the three stages on `s` (captured into the graph, or run directly while tuning).
static ufob_status batch_enqueue(ufob_batch *b, int variant, cudaStream_t s)
{
    const uint32_t n = (uint32_t)b->fjobs.size();
    const bool pairs = b->storage != UFOB_F32;
    UFOB_CUDA_TRY(cudaMemsetAsync(b->d_counters.ptr, 0, 2 * sizeof(uint32_t), s));
    k_batch_sincos<<<dim3((b->maxP + 255) / 256, n), 256, 0, s>>>(b->d_geo.as<double>(), b->d_rows.as<uint32_t>(),
                                                                 b->d_outs.as<float2 *>());
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    const int out_kind = !pairs ? 0 : (b->storage == UFOB_F16 ? 3 : 4);
    UFOB_TRY(filter_batch_launch(b->d_fjobs.as<BatchFilter>(), b->d_fitems.as<uint2>(), (uint32_t)b->fitems.size(),
                                 b->maxN, b->d_counters.as<uint32_t>(), out_kind, s));
    const SinoKind kind = !pairs ? SINO_F32 : (b->storage == UFOB_F16 ? SINO_F16_PAIRS : SINO_BF16_PAIRS);
    const bool kahan = pairs && b->maxP >= 1500;
    return bp_batch_launch(b->d_bjobs.as<BatchBP>(), b->d_bitems.as<uint2>(), (uint32_t)b->bitems.size(),
                           b->d_counters.as<uint32_t>() + 1, kind, kahan, variant, s);
}

// Build job descriptors, work lists and tensor maps for tile variant `v`.
static ufob_status batch_build(ufob_batch *b, const ufob_job *jobs, uint32_t n, int v)
{
    const bool pairs = b->storage != UFOB_F32;
    int tx, ty, winw;
    bp_batch_tile(v, &tx, &ty, &winw);
    b->fjobs.assign(n, BatchFilter{});
    b->bjobs.assign(n, BatchBP{});
    b->fitems.clear();
    b->bitems.clear();
    b->geo.assign(2 * n, 0.0);
    b->rows.assign(n, 0);
    b->outs.assign(n, nullptr);
    b->maxN = b->maxP = 0;
    // workspace layout: filtered rows of every job, then the angle tables
    size_t wbytes = 0, tbytes = 0;
    std::vector<size_t> woff(n), toff(n);
    std::vector<uint32_t> pitch(n), nfft(n);
    for (uint32_t j = 0; j < n; j++) {
        const ufob_job &J = jobs[j];
        nfft[j] = b->props.size_x ? b->props.size_x : next_pow2(J.width);
        pitch[j] = pairs ? round_up(J.width + 1, 4) : round_up(J.width, 4);
        woff[j] = wbytes;
        wbytes += ((size_t)pitch[j] * J.height * 4 + 255) / 256 * 256;
        toff[j] = tbytes;
        tbytes += ((size_t)J.height * sizeof(float2) + 255) / 256 * 256;
        b->maxN = std::max(b->maxN, nfft[j]);
        b->maxP = std::max(b->maxP, J.height);
    }
    UFOB_TRY(b->work.ensure(wbytes));
    UFOB_TRY(b->tables.ensure(tbytes));
    for (uint32_t j = 0; j < n; j++) {
        const ufob_job &J = jobs[j];
        FilterPlan &plan = b->plans[nfft[j]];  // default-constructed in place on first use
        UFOB_TRY(filter_plan_build(b->props, nfft[j], plan, 0));
        void *filt = b->work.as<char>() + woff[j];
        float2 *tab = reinterpret_cast<float2 *>(b->tables.as<char>() + toff[j]);
        BatchFilter &F = b->fjobs[j];
        F.in = J.d_sino;
        F.out = filt;
        F.tw = plan.d_twiddle.as<float2>();
        F.gains = plan.d_gains.as<float2>();
        F.width = J.width;
        F.rows = J.height;
        F.in_pitch = J.width;
        F.out_w = J.width;
        F.out_pitch = pitch[j];
        F.N = nfft[j];
        F.log2N = ilog2(nfft[j]);
        BatchBP &B = b->bjobs[j];
        const uint32_t elems = pairs ? J.width + 1 : J.width;
        UFOB_TRY(make_sino_map(&B.map, filt, elems, J.height, 1, pitch[j], (uint64_t)pitch[j] * J.height,
                               (uint32_t)winw, 1));
        B.args.P = J.height;
        B.args.nz = 1;
        B.args.roi_x = B.args.roi_y = 0;
        B.args.roi_w = B.args.roi_h = J.width;
        B.args.axis = J.axis_pos > 0.0 ? (float)J.axis_pos : (float)J.width / 2.0f;
        B.args.norm = (float)M_PI / (float)J.height;
        B.args.sincos = tab;
        B.args.out = J.d_out;
        B.args.err = device_error_word();
        B.tiles_x = (J.width + tx - 1) / tx;
        B.tiles_y = (J.width + ty - 1) / ty;
        b->geo[2 * j] = J.angle_offset;
        b->geo[2 * j + 1] = J.angle_step > 0.0 ? J.angle_step : M_PI / (double)J.height;
        b->rows[j] = J.height;
        b->outs[j] = tab;
    }
    // filter items grouped by FFT width (largest first); backprojection items
    // ordered by decreasing angle count (longest tiles first)
    std::vector<uint32_t> order(n);
    for (uint32_t j = 0; j < n; j++) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c) { return nfft[a] > nfft[c]; });
    for (uint32_t j : order)
        for (uint32_t p = 0; p < (jobs[j].height + 1) / 2; p++) b->fitems.push_back(make_uint2(j, p));
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t c) { return jobs[a].height > jobs[c].height; });
    for (uint32_t j : order)
        for (uint32_t t = 0; t < b->bjobs[j].tiles_x * b->bjobs[j].tiles_y; t++) b->bitems.push_back(make_uint2(j, t));
    // upload
    UFOB_TRY(b->d_fjobs.ensure(sizeof(BatchFilter) * n));
    UFOB_TRY(b->d_bjobs.ensure(sizeof(BatchBP) * n));
    UFOB_TRY(b->d_fitems.ensure(sizeof(uint2) * b->fitems.size()));
    UFOB_TRY(b->d_bitems.ensure(sizeof(uint2) * b->bitems.size()));
    UFOB_TRY(b->d_counters.ensure(2 * sizeof(uint32_t)));
    UFOB_TRY(b->d_geo.ensure(sizeof(double) * 2 * n));
    UFOB_TRY(b->d_rows.ensure(sizeof(uint32_t) * n));
    UFOB_TRY(b->d_outs.ensure(sizeof(float2 *) * n));
    UFOB_CUDA_TRY(cudaMemcpy(b->d_fjobs.ptr, b->fjobs.data(), sizeof(BatchFilter) * n, cudaMemcpyHostToDevice));
    UFOB_CUDA_TRY(cudaMemcpy(b->d_bjobs.ptr, b->bjobs.data(), sizeof(BatchBP) * n, cudaMemcpyHostToDevice));
    UFOB_CUDA_TRY(cudaMemcpy(b->d_fitems.ptr, b->fitems.data(), sizeof(uint2) * b->fitems.size(),
                             cudaMemcpyHostToDevice));
    UFOB_CUDA_TRY(cudaMemcpy(b->d_bitems.ptr, b->bitems.data(), sizeof(uint2) * b->bitems.size(),
                             cudaMemcpyHostToDevice));
    UFOB_CUDA_TRY(cudaMemcpy(b->d_geo.ptr, b->geo.data(), sizeof(double) * 2 * n, cudaMemcpyHostToDevice));
    UFOB_CUDA_TRY(cudaMemcpy(b->d_rows.ptr, b->rows.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    UFOB_CUDA_TRY(cudaMemcpy(b->d_outs.ptr, b->outs.data(), sizeof(float2 *) * n, cudaMemcpyHostToDevice));
    return UFOB_OK;
}

static std::string batch_signature(const ufob_batch *b, const ufob_job *jobs, uint32_t n)
{
    std::string s;
    char buf[160];
    snprintf(buf, sizeof buf, "%d:%u:", (int)b->storage, b->props.size_x);
    s += buf;
    for (uint32_t j = 0; j < n; j++) {
        snprintf(buf, sizeof buf, "%p,%p,%u,%u,%.17g,%.17g,%.17g;", (const void *)jobs[j].d_sino,
                 (const void *)jobs[j].d_out, jobs[j].width, jobs[j].height, jobs[j].axis_pos, jobs[j].angle_step,
                 jobs[j].angle_offset);
        s += buf;
    }
    return s;
}

// Shape key for the tuning cache: storage plus the sorted (width, angle bucket) multiset.
static std::string tune_key(const ufob_batch *b, const ufob_job *jobs, uint32_t n)
{
    std::vector<std::pair<uint32_t, uint32_t>> shapes;
    for (uint32_t j = 0; j < n; j++) shapes.emplace_back(jobs[j].width, (jobs[j].height + 127) / 128);
    std::sort(shapes.begin(), shapes.end());
    uint64_t h = 1469598103934665603ull;  // FNV-1a over the shapes
    for (auto &p : shapes) {
        h = (h ^ p.first) * 1099511628211ull;
        h = (h ^ p.second) * 1099511628211ull;
    }
    char buf[96];
    snprintf(buf, sizeof buf, "bp_batch:st%d:n%u:%016llx", (int)b->storage, n, (unsigned long long)h);
    return buf;
}

static ufob_status batch_autotune(ufob_batch *b, const ufob_job *jobs, uint32_t n, cudaStream_t s, int *best)
{
    const std::string key = tune_key(b, jobs, n);
    const char *tune = getenv("UFOB_TUNE");
    if (tune_lookup(key, best) && *best >= 0 && *best < bp_batch_variants()) return UFOB_OK;
    *best = 0;
    if (tune && strcmp(tune, "0") == 0) return UFOB_OK;
    cudaEvent_t e0, e1;
    UFOB_CUDA_TRY(cudaEventCreate(&e0));
    UFOB_CUDA_TRY(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    for (int v = 0; v < bp_batch_variants(); v++) {
        UFOB_TRY(batch_build(b, jobs, n, v));
        UFOB_TRY(batch_enqueue(b, v, s));  // warm-up
        UFOB_CUDA_TRY(cudaEventRecord(e0, s));
        UFOB_TRY(batch_enqueue(b, v, s));
        UFOB_CUDA_TRY(cudaEventRecord(e1, s));
        UFOB_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        UFOB_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) {
            best_ms = ms;
            *best = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tune_store(key, *best);
    return check_device_error_word(s);
}

extern "C" ufob_status ufob_batch_run(ufob_batch *b, const ufob_job *jobs, uint32_t n, void *stream)
{
    if (!b || (!jobs && n)) return fail(UFOB_ERR_INVALID, "batch_run: NULL argument");
    if (!n) return UFOB_OK;
    UFOB_TRY(ensure_device());
    for (uint32_t j = 0; j < n; j++) {
        const ufob_job &J = jobs[j];
        if (!J.d_sino || !J.d_out || !J.width || !J.height)
            return fail(UFOB_ERR_INVALID, "batch job %u: NULL pointer or empty sinogram", j);
        const uint32_t N = b->props.size_x ? b->props.size_x : next_pow2(J.width);
        if (N < J.width) return fail(UFOB_ERR_REQUISITION, "Specified size must be greater than or equal to input size");
        if (N > 8192) return fail(UFOB_ERR_UNSUPPORTED, "batch job %u: FFT width %u above 8192", j, N);
        if (((uintptr_t)J.d_sino & 15) || (J.width & 3))
            return fail(UFOB_ERR_INVALID, "batch job %u: rows must be 16-byte aligned (width multiple of 4)", j);
    }
    cudaStream_t s = (cudaStream_t)stream;
    const std::string sig = batch_signature(b, jobs, n);
    if (sig != b->signature || !b->exec) {
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        if (b->graph) {
            cudaGraphDestroy(b->graph);
            b->graph = nullptr;
        }
        int v = b->pinned;
        if (v < 0) UFOB_TRY(batch_autotune(b, jobs, n, s, &v));
        UFOB_TRY(batch_build(b, jobs, n, v));
        // capture the whole batch (counter resets + three persistent launches) once
        cudaStream_t cap;
        UFOB_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        UFOB_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        ufob_status st = batch_enqueue(b, v, cap);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (st != UFOB_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        b->graph = g;
        UFOB_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
        b->signature = sig;
        b->variant = v;
    }
    UFOB_CUDA_TRY(cudaGraphLaunch(b->exec, s));
    note_launch(3);
    return UFOB_OK;
}

extern "C" int ufob_batch_variant(ufob_batch *b) { return b ? b->variant : -1; }

extern "C" int ufob_batch_variants(void) { return bp_batch_variants(); }

extern "C" ufob_status ufob_batch_set_variant(ufob_batch *b, int variant)
{
    if (!b) return fail(UFOB_ERR_INVALID, "batch handle is NULL");
    if (variant < -1 || variant >= bp_batch_variants())
        return fail(UFOB_ERR_INVALID, "batch: tile variant %d outside [-1, %d]", variant, bp_batch_variants() - 1);
    if (variant != b->pinned) {
        b->pinned = variant;
        b->signature.clear();  // rebuild and recapture on the next run
    }
    return UFOB_OK;
}
