// cfg_noalloc.cu -- partition + bucket scatter for callers that cannot allocate.
//
// Some callers may not call cudaMalloc at all: plugins whose host framework hands
// out every byte of device memory from its own pool, and services that forbid
// allocation on their request path (cudaMalloc and cudaFree may synchronise the
// whole device, stalling every other stream's work).  cfg_partition_noalloc serves
// them: it partitions one small job's packed input into weak super k-mers bucketed
// by subgraph, like the first two kernels of cfg_run, but keeps its scratch
// (record cursor, error word, per-subgraph histogram and fill counters, the
// unbucketed records) in a file-scope device array instead of allocated buffers,
// and writes only to the output buffers the caller passes in.  It allocates
// nothing, host or device, and never synchronises.
//
// Limits and sharing:
//   - the scratch array is NOALLOC_SCRATCH_BYTES (8 MiB); every GPU that loads the
//     library keeps it until the process exits;
//   - the input may hold at most NOALLOC_MAX_BASES bases (one record per
//     (k-1)-mer position is the worst case, and that many must fit);
//   - every call on a device uses the same array: two calls whose work overlaps
//     on that GPU (different streams, or host threads) race and corrupt each
//     other's output.  Serialise them, e.g. on one stream.  Each call clears the
//     parts that must start at zero itself.
//   - the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, once per device, with that device current).
//   - a failure found on the device (a fragment past n_bases or shorter than k+1,
//     more records than the caller's buffer holds) makes the scatter write
//     CFG_NOALLOC_FAILED to *d_n_records and nothing else; the records and bucket
//     offsets of that call are then not valid.
#include "cuttlefish_gpu.h"
#include "cfg_device.cuh"
#include "cfg_internal.h"

#include <mutex>

namespace cfg {

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 8u << 20;
constexpr uint32_t NOALLOC_MAX_GRAPHS = 65536;
// layout: [misc 256 B][hist 8 B x 65536][inst 4 B x 65536][fill 4 B x 65536][flat records 8 B each]
constexpr size_t OFF_MISC = 0;
constexpr size_t OFF_HIST = 256;
constexpr size_t OFF_INST = OFF_HIST + 8ull * NOALLOC_MAX_GRAPHS;
constexpr size_t OFF_FILL = OFF_INST + 4ull * NOALLOC_MAX_GRAPHS;
constexpr size_t OFF_RECS = OFF_FILL + 4ull * NOALLOC_MAX_GRAPHS;
constexpr uint64_t NOALLOC_MAX_RECORDS = (NOALLOC_SCRATCH_BYTES - OFF_RECS) / 8;
constexpr uint64_t NOALLOC_MAX_BASES = NOALLOC_MAX_RECORDS;

static_assert(NOALLOC_MAX_BASES == CFG_NOALLOC_MAX_BASES, "the header states the input limit");

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

struct NoallocMisc {
    unsigned long long rec_cursor;
    uint32_t err;
};

// Bucketed placement of the flat records; the record count and the partition's error
// word are read on the device.  A failed partition, or more records than either the
// scratch array or the caller's buffer (cap) holds, scatters nothing and reports
// CFG_NOALLOC_FAILED as the record count.
__global__ void k_noalloc_scatter(const uint32_t* __restrict__ bucket_off, cfg_record* __restrict__ out,
                                  uint64_t cap, unsigned long long* __restrict__ n_out) {
    const NoallocMisc* misc = (const NoallocMisc*)(g_noalloc_scratch + OFF_MISC);
    const uint64_t* flat = (const uint64_t*)(g_noalloc_scratch + OFF_RECS);
    uint32_t* fill = (uint32_t*)(g_noalloc_scratch + OFF_FILL);
    const uint64_t n = misc->rec_cursor;
    const bool failed = misc->err != 0 || n > NOALLOC_MAX_RECORDS || n > cap;
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = failed ? (unsigned long long)CFG_NOALLOC_FAILED : n;
    if (failed) return;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = flat[i];
        const uint32_t g = rec_g(r);
        const uint32_t slot = atomicAdd(fill + g, 1u);
        out[bucket_off[g] + slot] = cfg_record{rec_pos(r), (uint8_t)rec_len(r), (uint8_t)(rec_ld(r) | (rec_rd(r) << 1)), (uint16_t)g};
    }
}

std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[256] = {};   // device address of the array, per device

// Once per device, with that device current: the device address of the scratch array.
int scratch_on(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (device < 0 || device >= 256) return CFG_ERR_BAD_INPUT;
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) { cudaGetLastError(); return CFG_ERR_CUDA; }
        g_scratch_ptr[device] = (unsigned char*)p;
    }
    *out = g_scratch_ptr[device];
    return CFG_OK;
}

}  // namespace

}  // namespace cfg

using namespace cfg;

extern "C" int cfg_partition_noalloc(int device, const cfg_params* p, const uint64_t* d_packed, uint64_t n_bases,
                                     const uint64_t* d_frag_off, const uint32_t* d_frag_len, uint64_t n_frags,
                                     cfg_record* d_records, uint64_t records_cap, uint32_t* d_bucket_off,
                                     uint64_t* d_n_records, void* stream) {
    if (!p || p->k < 3 || p->k > MAX_K || (p->k % 2) == 0 || p->l < 1 || p->l > 32 || p->l > p->k - 1) return CFG_ERR_BAD_INPUT;
    if (p->graph_count == 0 || p->graph_count > NOALLOC_MAX_GRAPHS || (p->graph_count & (p->graph_count - 1))) return CFG_ERR_BAD_INPUT;
    if (n_bases > NOALLOC_MAX_BASES) return CFG_ERR_BAD_INPUT;   // beyond the fixed scratch: refuse, never overflow
    if ((n_bases && !d_packed) || (n_frags && (!d_frag_off || !d_frag_len)) || !d_bucket_off || !d_n_records) return CFG_ERR_BAD_INPUT;
    if (records_cap < n_bases || (n_bases && !d_records)) return CFG_ERR_BAD_INPUT;   // room for the worst case
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) { cudaGetLastError(); return CFG_ERR_CUDA; }
    if (prev != device && cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return CFG_ERR_CUDA; }
    int rc = CFG_OK;
    unsigned char* s = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    do {
        rc = scratch_on(device, &s);
        if (rc) break;
        // the misc words, histogram and fill counters must start at zero
        if (cudaMemsetAsync(s, 0, OFF_RECS, st) != cudaSuccess) { rc = CFG_ERR_CUDA; break; }
        PartitionArgs a{};
        a.packed = d_packed; a.frag_off = d_frag_off; a.frag_len = d_frag_len;
        a.n_frags = n_frags; a.n_bases = n_bases;
        a.k = p->k; a.l = p->l; a.w = p->k - p->l;
        a.gmask = p->graph_count - 1;
        a.seed0 = wy_seed0_host();
        a.seg = 2048;
        a.recs = (uint64_t*)(s + OFF_RECS); a.rec_cap = NOALLOC_MAX_RECORDS;
        a.rec_cursor = &((NoallocMisc*)(s + OFF_MISC))->rec_cursor;
        a.hist = (unsigned long long*)(s + OFF_HIST);
        a.err = &((NoallocMisc*)(s + OFF_MISC))->err;
        if (n_bases) launch_partition(a, st);
        launch_bucket_scan((const unsigned long long*)(s + OFF_HIST), p->graph_count, d_bucket_off,
                           (uint32_t*)(s + OFF_INST), (uint32_t*)(s + OFF_FILL), st);
        k_noalloc_scatter<<<148 * 4, 256, 0, st>>>(d_bucket_off, d_records, records_cap, (unsigned long long*)d_n_records);
        if (cudaGetLastError() != cudaSuccess) { rc = CFG_ERR_CUDA; break; }
    } while (0);
    if (prev != device) cudaSetDevice(prev);
    return rc;
}
