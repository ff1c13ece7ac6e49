// noalloc.cu - the spreading operator without any device allocation.
//
// Some callers cannot let a library allocate device memory: a host program
// that owns the whole HBM budget through its own pool (a serving process, or
// an MD engine that reserves nearly all device memory up front) would see an
// allocation behind its back fail or push it over budget, and cudaMalloc /
// cudaFree synchronise the device, which a caller stepping in a tight loop
// cannot afford.  selm_op_spread_noalloc serves them: the caller passes
// device buffers for the inputs and the output, and the scratch the spread
// needs (the counting sort of monomers into 16x8x16-cell spread tiles) lives in one
// file-scope __device__ array of fixed size that every GPU loading this
// library holds until the process exits.
//
// The call accumulates: fgrid -= Lambda(tf), as selm_op_spread does; a caller
// that wants a fresh spread zeroes fgrid first.
//
// Limits: at most kNoAllocMaxAtoms monomers, kNoAllocMaxTiles spread tiles of
// 16x8x16 cells, ceil(nx/16)*ceil(ny/8)*ceil(nz/16) (128^3 uses 1024), and
// kNoAllocEntries tile entries per monomer (a monomer
// is filed under every tile its stencil reaches: at most 8 on grids whose
// tiles span at least 5 cells per axis), about 4.5 MB in all.  All calls
// share the one array, so calls whose work overlaps on the GPU (different streams, no ordering between them) race on
// it; order them on one stream or with events.  The array keeps the last
// call's contents; the parts that must start at zero (bucket counts, the
// large-bucket counter) are cleared on the caller's stream by every call.
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture.
#include <mutex>
#include <string>

#include "../../include/selm_b200.h"
#include "selm_engine.h"
#include "selm_kernels.h"

using namespace selm;

namespace {

constexpr int kNoAllocMaxAtoms = 65536;
constexpr int kNoAllocMaxTiles = 4096;
constexpr int kNoAllocEntries = 8;
constexpr long kScanTmp = 2 * ((kNoAllocMaxTiles + 1 + 4095) / 4096) + 2;
// counts, offsets (nbk+1 each), cursor, big_list (nbk each), big_count, scan temp, bucket_of (M),
// unsorted and sorted (kNoAllocEntries * M each)
constexpr long kScratchInts = 2L * (kNoAllocMaxTiles + 1) + 2L * kNoAllocMaxTiles + 1 + kScanTmp +
                              (1L + 2L * kNoAllocEntries) * kNoAllocMaxAtoms;

static __device__ __align__(256) int g_spread_scratch[kScratchInts];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
int* g_scratch_addr[kMaxDevices] = {nullptr};

int scratch_for_current_device(int** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return selm_fail(SELM_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_spread_scratch);
    if (e != cudaSuccess)
      return selm_fail(SELM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<int*>(p);
  }
  *out = g_scratch_addr[dev];
  return SELM_OK;
}

}  // namespace

extern "C" int selm_op_spread_noalloc(int precision, const int dims[3], double lo, double dx, void* fgrid, int natoms,
                                      const double* x, const double* tf, void* stream) {
  if (!dims) return selm_fail(SELM_ERR_INVALID, "dims is NULL");
  for (int a = 0; a < 3; a++)
    if (dims[a] < 4 || dims[a] > 1024) return selm_fail(SELM_ERR_INVALID, "dims must be in [4,1024]");
  if (precision != 64 && precision != 32) return selm_fail(SELM_ERR_INVALID, "precision must be 64 or 32");
  if (natoms < 0 || !fgrid || (natoms > 0 && (!x || !tf))) return selm_fail(SELM_ERR_INVALID, "bad buffers");
  if (natoms > kNoAllocMaxAtoms)
    return selm_fail(SELM_ERR_INVALID, "selm_op_spread_noalloc: more than 65536 monomers (the fixed scratch size)");
  const BinSpec bs = spread_bin_spec(dims, lo, dx);
  const long nbk = (long)bs.nb[0] * bs.nb[1] * bs.nb[2];
  if (nbk > kNoAllocMaxTiles)
    return selm_fail(SELM_ERR_INVALID, "selm_op_spread_noalloc: grid needs more than 4096 spread tiles of 16x8x16 cells "
                      "(ceil(nx/16)*ceil(ny/8)*ceil(nz/16); 128^3 uses 1024)");
  const long per = spread_entries_per_monomer(bs);
  if (per > kNoAllocEntries)
    return selm_fail(SELM_ERR_INVALID, "selm_op_spread_noalloc: grid tiles too small for the fixed scratch");
  if (natoms == 0) return SELM_OK;
  int* base = nullptr;
  int rc = scratch_for_current_device(&base);
  if (rc) return rc;
  BinBuffers bb{};
  int* q = base;
  bb.counts = q; q += nbk + 1;
  bb.offsets = q; q += nbk + 1;
  bb.cursor = q; q += nbk;
  bb.big_list = q; q += nbk;
  bb.big_count = q; q += 1;
  bb.scan_tmp = q; q += kScanTmp;
  bb.bucket_of = q; q += natoms;
  bb.unsorted = q; q += per * natoms;
  bb.sorted = q;
  CouplingArgs a{};
  a.nx = dims[0];
  a.ny = dims[1];
  a.nz = dims[2];
  a.lo = lo;
  a.dx = dx;
  a.M = natoms;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = bin_particles(x, natoms, bs, bb, st);
  if (e == cudaSuccess) {
    e = (precision == 64)
            ? spread_gather<double>(static_cast<double*>(fgrid), true, x, tf, bs, bb.offsets, bb.sorted, a, st)
            : spread_gather<float>(static_cast<float*>(fgrid), true, x, tf, bs, bb.offsets, bb.sorted, a, st);
  }
  if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("selm_op_spread_noalloc: ") + cudaGetErrorString(e));
  return SELM_OK;
}
