// Gate amplitudes without any device allocation.
//
// Some callers cannot call cudaMalloc: a host application whose device memory is owned end to end by its
// own allocator (a framework's caching allocator that has reserved the whole budget), a long-running
// service loop that must not pay the device-wide synchronisation cudaMalloc/cudaFree imply while other
// streams are busy, or a plug-in that is only handed buffers and is not allowed to allocate at all.  For
// them, dsg_gate_amps_noalloc computes what dsg_gate_amps computes -- the pre-gate and full-gate side
// amplitudes of explicit seeds -- with every intermediate (octave tables, counters, survivor lists, blur
// taps) in one fixed array of device memory that belongs to this library: g_noalloc_scratch below, sized
// for at most DSG_NOALLOC_MAX_SEEDS seeds (about 2.6 MB) and held by every GPU that loads the library
// until the process exits.  The caller passes device pointers for the seeds and both outputs.
//
// Set-up: the first call on each device resolves the array's device address (cudaGetSymbolAddress; in host
// code the array's name is only a host-side stand-in, never a device address) and computes the blur taps
// into it with one synchronous copy back; make that first call before any stream capture.  Every call
// shares the one array and leaves the previous call's contents in it; this file resets the counters that
// must start at zero on each call.  The set-up is kept for the life of the process: a cudaDeviceReset of a
// device after the first call there is not supported (the array's contents and address are not restored).  Calls whose work overlaps on the GPU (different streams, or several
// host threads at once) race on the array and must be serialised by the caller.
#include "common.cuh"
#include <mutex>

namespace dsg {
namespace gate {
void launch_amps_on(const uint64_t *d_seeds, uint32_t n, void *d_oct, uint32_t *d_counters, uint64_t *d_tmp_seeds, uint32_t *d_tmp_idx,
                    float *d_tmp_amp, float *d_pre, float *d_full, const float taps24[24], int pg_blocks, int fg_blocks, cudaStream_t st);
void gate_taps_into(float *d_out, cudaStream_t st);
size_t oct_bytes();
int pregate_blocks_per_sm();
int fullgate_blocks_per_sm();
}  // namespace gate

namespace {
constexpr uint32_t MAXS = DSG_NOALLOC_MAX_SEEDS;
// Scratch layout (byte offsets): counters | octave tables (2 per seed) | survivor seeds | indices | amps | taps
constexpr size_t OFF_CNT = 0, OFF_OCT = 256, OCT_BYTES = 304;
constexpr size_t OFF_SEEDS = OFF_OCT + size_t(2) * MAXS * OCT_BYTES, OFF_IDX = OFF_SEEDS + size_t(MAXS) * 8;
constexpr size_t OFF_AMP = OFF_IDX + size_t(MAXS) * 4, OFF_TAPS = OFF_AMP + size_t(MAXS) * 4, SCRATCH_BYTES = OFF_TAPS + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

struct PerDevice { bool ready = false; unsigned char *scratch = nullptr; float taps[24]; int pg_blocks = 0, fg_blocks = 0; };
constexpr int MAX_DEVICES = 64;
PerDevice g_dev[MAX_DEVICES];
std::mutex g_mu;

__global__ void k_reset_counters(uint32_t *c, uint32_t n) { c[0] = n; c[1] = 0; c[2] = n; c[3] = 0; }
}  // namespace
}  // namespace dsg

extern "C" int dsg_gate_amps_noalloc(const uint64_t *seeds, uint32_t n, float *pre, float *full, void *stream) {
    using namespace dsg;
    if (n > MAXS) { set_error("dsg_gate_amps_noalloc: %u seeds exceed the fixed scratch capacity of %u seeds per call", n, MAXS); return DSG_E_ARG; }
    if (n && (!seeds || !pre || !full)) { set_error("dsg_gate_amps_noalloc: null device pointer"); return DSG_E_ARG; }
    if (gate::oct_bytes() != OCT_BYTES) { set_error("dsg_gate_amps_noalloc: octave table layout mismatch"); return DSG_E_STATE; }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { set_error("dsg_gate_amps_noalloc: %s", cudaGetErrorString(e)); return DSG_E_CUDA; }
    if (dev < 0 || dev >= MAX_DEVICES) { set_error("dsg_gate_amps_noalloc: device %d out of range", dev); return DSG_E_ARG; }
    PerDevice &d = g_dev[dev];
    {
        std::lock_guard<std::mutex> l(g_mu);
        if (!d.ready) {                                  // once per device, with that device current
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) { set_error("dsg_gate_amps_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e)); return DSG_E_CUDA; }
            unsigned char *s = static_cast<unsigned char *>(p);
            (void)cudaGetLastError();                    // an error the caller left pending is not this set-up's
            gate::gate_taps_into(reinterpret_cast<float *>(s + OFF_TAPS), nullptr);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaMemcpy(d.taps, s + OFF_TAPS, sizeof d.taps, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) { set_error("dsg_gate_amps_noalloc: set-up: %s", cudaGetErrorString(e)); return DSG_E_CUDA; }
            int sms = 0;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) { set_error("dsg_gate_amps_noalloc: %s", cudaGetErrorString(e)); return DSG_E_CUDA; }
            d.pg_blocks = std::max(2, (gate::pregate_blocks_per_sm() * sms) & ~1);
            d.fg_blocks = std::max(2, (gate::fullgate_blocks_per_sm() * sms) & ~1);
            d.scratch = s;
            d.ready = true;
        }
    }
    if (!n) return DSG_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char *s = d.scratch;
    uint32_t *cnt = reinterpret_cast<uint32_t *>(s + OFF_CNT);
    (void)cudaGetLastError();                            // report only this call's launch errors below
    k_reset_counters<<<1, 1, 0, st>>>(cnt, n);
    gate::launch_amps_on(seeds, n, s + OFF_OCT, cnt, reinterpret_cast<uint64_t *>(s + OFF_SEEDS), reinterpret_cast<uint32_t *>(s + OFF_IDX),
                         reinterpret_cast<float *>(s + OFF_AMP), pre, full, d.taps, d.pg_blocks, d.fg_blocks, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) { set_error("dsg_gate_amps_noalloc: launch: %s", cudaGetErrorString(e)); return DSG_E_CUDA; }
    return DSG_OK;
}
