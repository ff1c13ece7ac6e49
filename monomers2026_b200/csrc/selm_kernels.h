// selm_kernels.h - host-side launchers of the SELM device kernels (internal).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace selm {

// kernels launched by this library since load (process-wide, host side)
void count_launches(unsigned n);
void uncount_launches(unsigned long long n);  // launches recorded into a graph capture, not run
unsigned long long launches_total();

constexpr int kSumParts = 296;  // fixed number of partial sums (2 per SM)

// Twiddle tables of the three axes, forward (sign -1) and backward (+1).
template <typename T> struct FftTables {
  FftRadix rx, ry, rz;
  const cpx<T>*wx_f, *wx_b, *wy_f, *wy_b, *wz_f, *wz_b;
};

// ---- fluid, reference structure (FP64)
cudaError_t plain_fluid_run(const double* u_old, double* u_new, const double* f, double* p, double2* work,
                            double* partial, double* sum, int nx, int ny, int nz, double dx, double dt, double mu,
                            double rho, const FftTables<double>& tb, cudaStream_t st);
cudaError_t plain_compute_f(double* f, double2* work, int nx, int ny, int nz, double dx, double kB, double T,
                            double dt, double mu, bool stochastic, uint64_t seed, uint64_t step, int noise_mode,
                            const FftTables<double>& tb, cudaStream_t st);
template <typename T>
cudaError_t fft3_r2c(const T* in, cpx<T>* out, int nx, int ny, int nz, int ncomp, const FftTables<T>& tb,
                     cudaStream_t st);
template <typename T>
cudaError_t fft3_c2r(cpx<T>* in, T* out, int nx, int ny, int nz, int ncomp, T scale, const FftTables<T>& tb,
                     cudaStream_t st);

// ---- binning (counting sort of monomers into buckets, deterministic order)
struct BinSpec {
  int mode;      // 0: grid tiles (cell = floor((x-lo)/dx), bucket = cell / tile), 1: cells of size L/nc,
                 // 2: spread tiles (a monomer in every tile its union stencil reaches)
  int n[3];      // grid points (mode 0) or cells (mode 1) per axis
  int tile[3];   // tile extent in grid cells (mode 0), 1 in mode 1
  int nb[3];     // buckets per axis
  double lo, dx, L;
};
struct BinBuffers {
  int* counts;    // [nbuckets + 1]
  int* offsets;   // [nbuckets + 1]
  int* cursor;    // [nbuckets]
  int* bucket_of; // [M]
  int* unsorted;  // [M]
  int* sorted;    // [M]
  int* scan_tmp;  // [scan_tmp_size(nbuckets)]
  int* big_list;  // [nbuckets] buckets too large for one warp
  int* big_count; // [1]
};
long scan_tmp_size(long n);
// spread tiles (mode 2): every monomer filed under each tile its stencil reaches
BinSpec spread_bin_spec(const int dims[3], double lo, double dx);
long spread_entries_per_monomer(const BinSpec& bs);
// rec_b (optional, mode 2): stencil bases of a per-monomer record (ints b[axis][shift]
// at the record's start), rec_stride ints apart; without it the bases come from x
cudaError_t bin_particles(const double* x, int M, const BinSpec& bs, const BinBuffers& bb, cudaStream_t st,
                          const int* rec_b = nullptr, int rec_stride = 0);

// ---- coupling and monomer update
// Per-monomer stencil of one step: wrapped base cell of the 4-point stencil and
// its weight factors, per axis, unshifted and shifted by half a cell.
// Spread-tile slots filled during the interpolation (no counting sort): the
// candidates of tile t sit at slots[t*cap .. t*cap + min(count[t], cap)), the
// ones beyond a tile's capacity in the overflow list.  The spread clears
// count[] and the overflow counter for the next step.
struct TileSlots {
  int* count = nullptr;       // [ntiles] appended so far
  int* slots = nullptr;       // [ntiles][cap]
  int cap = 0;
  int2* ovf = nullptr;        // (tile, monomer) beyond a tile's capacity
  int* ovf_count = nullptr;   // [1]
  int ovf_cap = 0;
  unsigned* done = nullptr;   // [1] spread blocks finished; the last one resets ovf_count
  BinSpec bs{};               // the spread tiles (mode 2)
  // home mode (FP32 grids): a monomer is filed once, under the tile of its
  // cell floor((x - lo)/dx); the spread accumulates each tile's monomers into
  // a box of the tile plus a 2-cell halo, written to box[] (zeros for a tile
  // without monomers), and a fold pass sums the boxes that cover each cell.
  // live[t] = tile t had monomers.
  // The interpolation also leaves, per tile, the largest |impulse| of its
  // monomers (tmax: the bits of the FP64 value, which order as unsigned
  // integers for non-negative values, NaN above all) and whether a weight
  // factor above 1/2 occurred (quirk: the reference's distance-2 factor of 1),
  // the scale of the tile's fixed-point box; the spread clears both.
  int home = 0;
  float* box = nullptr;       // [ntiles][3][tile z + 4][tile y + 4][tile x + 4]
  int* live = nullptr;        // [ntiles]
  unsigned long long* tmax = nullptr;  // [ntiles]
  int* quirk = nullptr;                // [ntiles]
  // z-slab of a decomposed instance: monomers are filed only under tiles of
  // the layers [tz0, tz1) (tz1 == 0: all), the spread's block b takes tile
  // tile0 + b, and the grid it writes holds planes z0.. with components
  // cstride apart (0: the whole grid's N)
  int tz0 = 0, tz1 = 0, tile0 = 0, z0 = 0;
  long cstride = 0;
};
template <typename T> struct alignas(16) WRec {
  T w[3][2][4];  // weight factors [axis][unshifted, shifted][point] (16-byte aligned rows)
  int b[3][2];   // stencil bases wrapped into [0, n): [axis][unshifted, shifted]
  // home mode: per component, the slot of its stencil base in the home tile's
  // box (the tile plus 2 cells on each side, x fastest), without the component offset
  unsigned short hs[3];
};
// the bases of record 0 and the record stride in ints, for the binning kernels
template <typename T> inline const int* wrec_bases(const WRec<T>* rec) {
  return reinterpret_cast<const int*>(reinterpret_cast<const char*>(rec) + offsetof(WRec<T>, b));
}
template <typename T> constexpr int wrec_stride() {
  static_assert(sizeof(WRec<T>) % sizeof(int) == 0, "record size");
  return (int)(sizeof(WRec<T>) / sizeof(int));
}
struct CouplingArgs {
  int nx, ny, nz;
  double lo, hi, dx, dt, upsilon, coef;
  int stochastic;
  uint64_t seed, step;
  const uint64_t* step_ptr;  // if set, the step index is read on the device (graph replay)
  int M;
};
template <typename T>
cudaError_t interp_update(const T* u, const double* x_old, double* x_new, double* v, double* f, const double* m,
                          double* tf, const int* order, WRec<T>* rec, const CouplingArgs& a, uint32_t* err,
                          cudaStream_t st, const TileSlots* ts = nullptr);
// decomposed instance: the slab's part of the interpolation, and the update
// from the interpolation summed over the slabs
template <typename T>
cudaError_t interp_partial(const T* u_slab, const double* x, const CouplingArgs& a, int z0, int nzl, T* out,
                           cudaStream_t st);
template <typename T>
cudaError_t interp_update_gathered(const T* gathered, const double* x_old, double* x_new, double* v, double* f,
                                   const double* m, double* tf, WRec<T>* rec, const CouplingArgs& a, uint32_t* err,
                                   cudaStream_t st, const TileSlots& ts);
template <typename T>
cudaError_t interp_only(const T* u, const double* x, int M, int nx, int ny, int nz, double lo, double dx, double* out,
                        cudaStream_t st);
cudaError_t spread_prepare_attributes();
// staged monomer upload: check the staged positions (cnt[2] on the device),
// then commit positions and velocities (vin NULL: zeros) if both counts are 0
cudaError_t stage_check(const double* xin, long n, double lo, double hi, double lim, unsigned long long* cnt,
                        cudaStream_t st);
cudaError_t stage_commit(const double* xin, const double* vin, double* x, double* v, long n,
                         const unsigned long long* cnt, cudaStream_t st);
template <typename T>
cudaError_t spread_gather(T* fgrid, bool accumulate, const double* x_old, const double* tf, const BinSpec& bs,
                          const int* offsets, const int* sorted, const CouplingArgs& a, cudaStream_t st,
                          const WRec<T>* rec = nullptr);

template <typename T>
cudaError_t spread_slots(T* fgrid, bool accumulate, const double* x_old, const double* tf, const TileSlots& ts,
                         const CouplingArgs& a, cudaStream_t st, const WRec<T>* rec);

// ---- conservative forces (FP64)
// quasi-steady form: stencil records at x and tf = -F inv_dv before the
// spread; v = Gamma u (x_old), x_new = x_old + dt v after the fluid solve
template <typename T>
cudaError_t qs_prepare(const double* x, const double* f, double* tf, WRec<T>* rec, const CouplingArgs& a,
                       double inv_dv, cudaStream_t st, const TileSlots* ts, uint32_t* err);
template <typename T>
cudaError_t qs_move(const T* u, const double* x_old, double* x_new, double* v, const CouplingArgs& a, uint32_t* err,
                    cudaStream_t st);

struct ForceTopo {
  int M, ntypes;
  const int* type;        // [M] 1-based
  int bond_style;         // 0 none 1 harmonic 2 fene
  const int* bond_off;    // [M+1] CSR of incident bonds
  const int* bond_nbr;    // partner atom
  const int* bond_typ;    // bond type
  const double* bond_coeff;  // [ntb+1][4]
  int angle_style;        // 0 none 1 harmonic
  const int* ang_off;     // [M+1] CSR of incident angles
  const int* ang_atoms;   // [nentries][4] = type, i, j, k (0-based)
  const double* angle_coeff;  // [nta+1][2]
  int pair_style;         // 0 none 1 lj/cut
  const double* pair_coeff;  // [(nt+1)^2][3] eps sigma rc
  const int* sp_off;      // [M+1] CSR of special partners
  const int* sp_nbr;
  const double* sp_w;     // weight per entry
  double body[3];
  double lo, hi;
  double rc2max;          // largest pair cutoff squared (quick reject)
};
// Verlet neighbour list of the pair style: every partner j within
// rl = (largest cutoff + skin) of i, pairs of special weight 0 left out,
// sorted by j.  Rebuilt from the force cells when some monomer has moved more
// than skin/2 since the last build (minimum image), which keeps every pair
// within the cutoff on the list.
struct NeighborList {
  int cap = 0;             // entries per monomer
  int* idx = nullptr;      // [cap][M]: partner j | weight class << 30
  int* cnt = nullptr;      // [M]
  double* xb = nullptr;    // [3M] positions at the last build
  double* xs = nullptr;    // [3M] positions in cell order (slot of the cell sort), for the build
  int* flag = nullptr;     // rebuild requested: set by the check, cleared by the forces kernel
  double rl2 = 0.0;        // list radius squared
  double half_skin2 = 0.0; // (skin / 2)^2
  double wtab[4] = {1.0, 1.0, 1.0, 1.0};  // pair weight by class: 1, special_lj[0..2]
};
// check displacements and, where needed, rebuild (every kernel returns at
// once when no rebuild is due, so the launch sequence is the same every step)
cudaError_t neighbor_update(const double* x, const ForceTopo& t, const BinSpec& cells, const BinBuffers& bb,
                            const NeighborList& nl, uint32_t* err, cudaStream_t st);
// bonds, angles, pairs from the list (nl may be null without a pair style), body force
cudaError_t compute_forces(const double* x, double* f, const ForceTopo& t, const NeighborList* nl, uint32_t* err,
                           cudaStream_t st);
// exclusive scan over n ints; when flag is non-null the kernels return at once while *flag == 0
cudaError_t exclusive_scan(const int* in, int* out, long n, int* tmp, cudaStream_t st, const int* flag = nullptr);

}  // namespace selm
