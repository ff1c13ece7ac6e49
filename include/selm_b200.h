/*
 * selm_b200.h - C ABI of libselm_b200.so, the B200-native SELM
 * fluctuating-hydrodynamics step (monomers coupled to a periodic Stokes
 * fluid through the Peskin 4-point kernel).
 *
 * The reference (yaohong99/monomers2026, data/src/selm-main/src/cuda) is an
 * executable whose plugin surface is a C++ lifecycle:
 *   Selm{initial, run, compute_f, final}            cuda/SELM.cuh:22-27
 *   Eulerian{initial, compute_f, run, final}        cuda/SELM_Eulerian.cuh:23-27
 *   Lagrangian{initial, compute_f, run, final}      cuda/SELM_Lagrangian.cuh:41-47
 * with state shared through public pointers (d_u, d_f, dim, dx, d_x, d_v,
 * d_f, d_m, lo, hi).  This header is that surface as plain C: an opaque
 * handle, FP64 host buffers that are copied (never aliased), and int status
 * codes instead of exit(-1) (cuda/check.cuh:6-10).
 *
 * Conventions: particles are AoS [M][3] doubles; grid fields are planar
 * [3][Nz][Ny][Nx] doubles with n = (k*Ny + j)*Nx + i, exactly the
 * reference's layout.  All calls return SELM_OK (0) on success; on failure
 * selm_last_error() describes the most recent error of the calling thread.
 */
#ifndef SELM_B200_H
#define SELM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SELM_OK 0
#define SELM_ERR_INVALID 1   /* bad argument or size */
#define SELM_ERR_CUDA 2      /* CUDA runtime error */
#define SELM_ERR_STATE 3     /* call out of lifecycle order */
#define SELM_ERR_NOMEM 4     /* device allocation failed or over budget */
#define SELM_ERR_IO 5        /* input file missing or malformed */
#define SELM_ERR_NUMERIC 6   /* the device error word is non-zero */

/* form of the step */
#define SELM_FORM_PLAIN64 0  /* reference structure, FP64 (drop-in) */
#define SELM_FORM_FUSED64 1  /* spectral state, fused pencil FFT kernels, FP64 */
#define SELM_FORM_FUSED32 2  /* same in FP32 with FP64 positions, zero mode and noise prefactor */

#define SELM_INTEGRATOR_INERTIAL 0     /* reference scheme (cuda/SELM_Kernel.cu:155-195,302-373) */
/* Overdamped form, no counterpart in the reference (fused forms only):
 * u = P (F_hat / dV + g_hat) / (mu lambda_h) with the conservative forces F
 * spread at x^n and thermal forcing of variance 2 kB T mu lambda_h / (dt dV)
 * per mode; v = Gamma u (x^n), x^{n+1} = x^n + dt v; f keeps the
 * conservative force. */
#define SELM_INTEGRATOR_QUASI_STEADY 1

#define SELM_NOISE_REF_COMPAT 0 /* reference draw: x=0 and x=Nx/2 planes Hermitian-averaged by the c2r */
#define SELM_NOISE_EXACT 1      /* Hermitian-correct draw: full variance on those planes */

/* device error word bits (selm_status) */
#define SELM_STATUS_NONFINITE 0x1u
#define SELM_STATUS_DISPLACEMENT 0x2u /* |v dt| > L/2: the reference only prints (cuda/SELM_Kernel.cu:363) */
#define SELM_STATUS_FENE_STRETCH 0x4u
#define SELM_STATUS_FENE_BROKEN 0x8u
#define SELM_STATUS_NLIST_OVERFLOW 0x20u /* a monomer had more pair partners in reach than its neighbour list holds */
#define SELM_STATUS_COPY_TIMEOUT 0x40u /* an asynchronous copy into shared memory did not complete within its bound; the step's fluid result is invalid */

/* Model.SELM keys (cuda/SELM.cu:17-48) plus the box and dt that the
 * reference takes from LAMMPS (domain->boxlo/hi, update->dt). */
typedef struct selm_params {
  int num_mesh_pts[3];       /* numMeshPtsPerDir (all equal, as the reference assumes), in [4, 1024]
                                with no prime factor above 61 (the FFT's radices) */
  double box_lo, box_hi;     /* cubic periodic box; dx = (hi - lo)/Nx */
  double rho, mu, KB, T, dt; /* rho mu KB T, timestep */
  int flag_stochastic;       /* flagStochasticDriving */
  unsigned long long seed;   /* SELM_Seed */
  int form;                  /* SELM_FORM_* */
  int integrator;            /* SELM_INTEGRATOR_* */
  int noise_mode;            /* SELM_NOISE_* */
} selm_params;

/* Force field of the LAMMPS-script subset the inputs use
 * (bond_style harmonic|fene, angle_style harmonic, pair_style lj/cut,
 * special_bonds lj weights, a uniform body force). Atom indices 0-based,
 * types 1-based as in LAMMPS data files. */
#define SELM_BOND_NONE 0
#define SELM_BOND_HARMONIC 1 /* coeff per type: K r0            (E = K (r-r0)^2) */
#define SELM_BOND_FENE 2     /* coeff per type: K R0 eps sigma  (LAMMPS bond_style fene) */
#define SELM_ANGLE_NONE 0
#define SELM_ANGLE_HARMONIC 1 /* coeff per type: K theta0(deg) (E = K (theta-theta0)^2) */
#define SELM_PAIR_NONE 0
#define SELM_PAIR_LJCUT 1 /* coeff per type pair (i,j) at (i*(ntypes+1)+j)*3: eps sigma rc */

typedef struct selm_topology {
  int natoms, ntypes;
  const int* type;            /* [natoms] */
  int nbonds, bond_style, nbondtypes;
  const int* bonds;           /* [nbonds][3] = type, i, j */
  const double* bond_coeff;   /* [(nbondtypes+1)][4] */
  int nangles, angle_style, nangletypes;
  const int* angles;          /* [nangles][4] = type, i, j(center), k */
  const double* angle_coeff;  /* [(nangletypes+1)][2] */
  int pair_style;
  const double* pair_coeff;   /* [(ntypes+1)^2][3] */
  double special_lj[3];       /* 1-2, 1-3, 1-4 weights (LAMMPS default 0 0 0) */
  double body_force[3];
} selm_topology;

typedef struct selm_sim selm_sim;

/* Host force provider, the role LAMMPS plays in the reference
 * (Lagrangian_LAMMPS::compute_f, cuda/SELM_Lagrangian_LAMMPS.cu:107-130):
 * called once per step with the new positions/velocities; f arrives zeroed,
 * so the provider may add into it or leave atoms without force untouched. */
typedef int (*selm_force_fn)(void* user, int natoms, const double* x, const double* v, double* f);

/* ---- lifecycle (Selm::Selm / initial / run / final) ---- */
/* replaces Selm::Selm() + Eulerian_Period::initial allocations (cuda/SELM.cu:17-48,
 * cuda/SELM_Eulerian_Period.cu:14-76) */
int selm_create(const selm_params* params, selm_sim** out);
/* replaces Selm::Selm() reading Model.SELM + LAMMPS script/data from a case
 * directory (cuda/SELM.cu:20, cuda/SELM_Lagrangian_LAMMPS.cu:21-28) */
int selm_create_from_files(const char* case_dir, selm_sim** out);
/* monomer state: replaces Lagrangian_LAMMPS::initial uploads (cuda/SELM_Lagrangian_LAMMPS.cu:71-93).
 * v NULL: zero velocities.  mass NULL: keep the masses of an earlier call (the
 * first call must give them), as the per-step round trip of a host force
 * provider moves positions and velocities only.  A non-finite position, or
 * one more than 1e6 box lengths away, or a non-positive mass returns
 * SELM_ERR_INVALID and leaves the monomers as they were; positions outside
 * the box are moved by whole box lengths into [lo, hi).  After the first call
 * the positions are checked on the device (staging buffers, 48 bytes per
 * monomer, allocated by the second call); the call returns once the host
 * buffers have been read and checked, with the update of the state queued on
 * the simulation's stream ahead of every later call. */
int selm_set_particles(selm_sim* s, int natoms, const double* x, const double* v, const double* mass);
/* device force field (replaces the per-step LAMMPS round trip) */
int selm_set_topology(selm_sim* s, const selm_topology* topo);
/* host force provider instead of the device force field */
int selm_set_force_callback(selm_sim* s, selm_force_fn fn, void* user);
/* Selm::initial (cuda/SELM.cu:55-58): initial forces, u = 0, first noise */
int selm_initial(selm_sim* s);
/* nsteps iterations of the body of Selm::run (cuda/SELM.cu:73-90) */
int selm_step(selm_sim* s, int nsteps);
/* Selm::final + destructor (cuda/SELM.cu:50-63) */
int selm_destroy(selm_sim* s);

/* ---- state access (the reference's public pointers, copied) ---- */
/* Positions, velocities and forces after the last step (any may be NULL).
 * Returns once they are in host memory.  Right after a step of a fused form
 * with the device force field, that is as soon as the step has written them:
 * the rest of that step (spread and fluid solve) may still run on the device
 * (selm_synchronize waits for it); every later call is ordered after it. */
int selm_get_particles(selm_sim* s, double* x, double* v, double* f);
/* Page-lock host arrays the caller owns (e.g. LAMMPS' atom->x, atom->v,
 * atom->f after each reallocation) so that the per-step copies above run as
 * direct transfers (about 50 GB/s here) rather than through pageable staging
 * (about 19 GB/s).  The caller unregisters before freeing the memory.
 * Registering a range that is already wholly page-locked is not an error; a
 * range that overlaps an earlier registration only in part (an array grown
 * in place) returns SELM_ERR_STATE: unregister the old range first.
 * selm_host_unregister undoes whatever registration starts at ptr, also one
 * made by another component of the process (cudaHostUnregister). */
int selm_host_register(void* ptr, unsigned long long bytes);
int selm_host_unregister(void* ptr);
/* t_f of the last inertial step, per monomer and component: the coupling
 * impulse -upsilon (v - Gamma u) dt plus the thermal kick, before the
 * conservative force is added (cuda/SELM_Kernel.cu:302-373).  The reference
 * writes (t_f + dt f_before) / dt to particleF.dat, the force array as the
 * update leaves it, before LAMMPS recomputes it
 * (mpi/SELM_Lagrangian_LAMMPS.cpp:79-82,280-300).  dt (the timestep) may be
 * NULL.  The quasi-steady form has no such impulse (SELM_ERR_STATE, dt still
 * set). */
int selm_get_coupling_impulse(selm_sim* s, double* tf, double* dt);
#define SELM_FIELD_U 0 /* Eulerian::d_u[cur_u] */
#define SELM_FIELD_F 1 /* Eulerian::d_f (forcing for the next fluid update) */
int selm_get_field(selm_sim* s, int which, double* out);       /* [3][Nz][Ny][Nx] */
int selm_set_field(selm_sim* s, int which, const double* in);
int selm_get_info(selm_sim* s, int* natoms, int dims[3], unsigned long long* step);
int selm_status(selm_sim* s, unsigned int* error_word);

/* ---- streams and timing ---- */
int selm_set_stream(selm_sim* s, void* cuda_stream); /* NULL = library-owned stream */
void* selm_get_stream(selm_sim* s);
int selm_synchronize(selm_sim* s);
/* per-kernel CUDA-event timing on the library stream */
int selm_profile_enable(selm_sim* s, int enable);
int selm_profile_read(selm_sim* s, const char* kernel, double* total_ms, long* launches);

/* ---- operator entry points on host buffers (unit-level parity) ---- */
/* gamma(): cuda/SELM_Kernel.cu:375-422 with the staggering of :328-338 */
int selm_op_interp(int precision, const int dims[3], double lo, double dx, const double* u, int natoms,
                   const double* x, double* out);
/* lambda(): cuda/SELM_Kernel.cu:424-470; fgrid -= Lambda(tf) */
int selm_op_spread(int precision, const int dims[3], double lo, double dx, double* fgrid, int natoms,
                   const double* x, const double* tf);
/* The spreading operator for callers that cannot let a library allocate device
 * memory (a host that owns the whole HBM budget through its own pool, or one
 * that cannot afford the device synchronisation cudaMalloc/cudaFree bring).
 * No counterpart in the reference.  Inputs and output are DEVICE pointers
 * (fgrid is double* for precision 64, float* for 32; x and tf are [M][3]
 * doubles); the call is ordered on `stream` (NULL = the legacy default stream).
 * It accumulates, fgrid -= Lambda(tf), as selm_op_spread does: zero fgrid
 * first for a fresh spread.  Scratch is a fixed file-scope device array
 * (about 4.5 MB): at most 65536 monomers and 4096 spread tiles of 16x8x16
 * cells, ceil(nx/16)*ceil(ny/8)*ceil(nz/16) (128^3 uses 1024); larger sizes
 * are rejected.  Calls that
 * overlap on the GPU share that array and race.  The first call on a device
 * looks up the array's address; make it before any stream capture. */
int selm_op_spread_noalloc(int precision, const int dims[3], double lo, double dx, void* fgrid, int natoms,
                           const double* x, const double* tf, void* stream);
/* cufftExecD2Z / cufftExecZ2D (cuda/SELM_Eulerian_Period.cu:113,117), unnormalised;
 * precision 64 or 32; half spectrum as interleaved complex doubles */
int selm_op_fft3_r2c(int precision, const int dims[3], const double* in, double* out);
int selm_op_fft3_c2r(int precision, const int dims[3], const double* in, double* out);

/* ---- batches: many simulations stepped by one graph launch ----
 * The reference runs one instance per process (cuda/main.cu:5-12, Selm::run
 * cuda/SELM.cu:70-98); these entry points replace running that executable
 * once per replica.  A batch steps fused-form simulations of any grid size and
 * monomer count together: each member's captured step graph becomes a child
 * of one graph, launched once per step on the batch's stream.  Members run on
 * the batch's stream while they belong to it (their own stream comes back when
 * they leave), are stepped only through the batch, and give the same results
 * bit for bit as when stepped alone.  Joining and leaving take effect at the
 * next selm_batch_step (the batch graph is rebuilt then). */
typedef struct selm_batch selm_batch;
int selm_batch_create(void* stream /* NULL: the batch owns a stream */, selm_batch** out);
int selm_batch_add(selm_batch* b, selm_sim* s);    /* s initialised, fused form, no host force callback */
int selm_batch_remove(selm_batch* b, selm_sim* s); /* waits for the batch's work */
int selm_batch_step(selm_batch* b, int nsteps);    /* asynchronous, like selm_step */
int selm_batch_size(selm_batch* b);
/* Serving (the reference serves one job per process, cuda/main.cu:5-12).
 * A job is a member with a step budget: it is stepped by the next nsteps
 * calls of selm_batch_step and then leaves the step graphs.
 * selm_batch_poll lists, without waiting, up to cap jobs whose budget is
 * spent and whose last step has finished on the device (*ndone of them).
 * selm_batch_retire removes such a job and reads back its x, v, f (any may
 * be NULL) on the job's own stream, without waiting for the batch's later
 * steps; SELM_ERR_STATE if its budget is not spent.  The simulation is not
 * destroyed. */
int selm_batch_add_job(selm_batch* b, selm_sim* s, long long nsteps);
int selm_batch_poll(selm_batch* b, selm_sim** done, int cap, int* ndone);
int selm_batch_retire(selm_batch* b, selm_sim* s, double* x, double* v, double* f);
void* selm_batch_get_stream(selm_batch* b);
int selm_batch_synchronize(selm_batch* b);
int selm_batch_destroy(selm_batch* b); /* members leave (not destroyed) */
/* device memory this simulation holds (for admission against an HBM budget);
 * the reference allocates per object in initial() (cuda/SELM_Eulerian_Period.cu:33-60) */
int selm_device_bytes(selm_sim* s, unsigned long long* bytes);

/* ---- tuning knobs of the fused forms (no counterpart in the reference) ----
 * SELM_TUNE_FFT_SPLIT: 0 = four-step FFT split with the largest factor <= 16,
 *   1 = the most balanced split (the same for sizes with one split);
 * SELM_TUNE_Z_BLOCKS: blocks per SM of the z-pencil kernel, 0 = as many as fit.
 * selm_tune_set changes one simulation (its step graph is recaptured);
 * selm_tune_default sets the value that simulations created later with this
 * cubic grid size and precision (32 or 64) start from.  monomers2026_b200's
 * autotuner times the candidates and records its choices with it. */
#define SELM_TUNE_FFT_SPLIT 1
#define SELM_TUNE_Z_BLOCKS 2
int selm_tune_set(selm_sim* s, int knob, int value);
int selm_tune_get(selm_sim* s, int knob, int* value);
int selm_tune_default(int grid, int precision, int knob, int value);

/* ---- trajectory output: DCD as written by LAMMPS' "dump ... dcd" ----
 * The reference's cases dump positions through LAMMPS
 * (cuda/SELM_Lagrangian_LAMMPS.cu:125-127 runs LAMMPS' output; the case
 * scripts hold "dump 1 all dcd N file").  Header, title, atom count, then per
 * frame the unit cell and X, Y, Z as float32; the header's frame count and
 * last step are kept current. */
typedef struct selm_dcd selm_dcd;
int selm_dcd_open(const char* path, int natoms, double dt, int first_step, int interval, const double box_len[3],
                  selm_dcd** out);
/* the same for a simulation: its monomer count, timestep, box, and its step as the first */
int selm_dcd_open_sim(const char* path, selm_sim* s, int interval, selm_dcd** out);
int selm_dcd_write(selm_dcd* d, const double* x /* host [natoms][3] */);
int selm_dcd_write_sim(selm_dcd* d, selm_sim* s); /* the simulation's current positions */
int selm_dcd_close(selm_dcd* d);
/* the case directory's "dump ID group dcd N file": N (0 if none) and the file */
int selm_case_dump(selm_sim* s, int* every, char* file, int len);

/* ---- on-device analysis: MSD, S(q), kinetic energy per direction ----
 * Replaces the reference's post-processing of DCD trajectories
 * (data/src/Diffusion Coefficient/MSD.py:14-91, fit of get_K.py) for runs
 * that should not write trajectories.  Each selm_analysis_sample records the
 * simulation's current positions as a float32 frame (what a DCD holds) and
 * adds, on the simulation's stream and without a host sync:
 *   MSD   lags l*lag_stride frames, l = 1..nlag: per direction the sum over
 *         frame pairs (n, n + lag) and monomers of the displacement folded
 *         once by the box (MSD.py:59-66), squared; MSD(l) = (sum of the three
 *         directions) / pairs[l]
 *   S(q)  |sum_j exp(i 2 pi n.x_j / L)|^2 / M for the nq integer triples n
 *   K_d   sum_j m_j v_jd^2 (equipartition: mean K_d / M = kT per direction)
 * Sums are deterministic (fixed reduction order).  An analysis belongs to
 * its simulation; destroying the simulation releases the analysis' device
 * memory (the handle must still be destroyed). */
typedef struct selm_analysis selm_analysis;
int selm_analysis_create(selm_sim* s, int nlag, int lag_stride, int nq, const int* qvec /* [nq][3] */,
                         selm_analysis** out);
int selm_analysis_sample(selm_analysis* a);
/* sums [nlag][3]; pairs [nlag] = (frame pairs) x monomers */
int selm_analysis_msd(selm_analysis* a, double* sums, long long* pairs);
/* per wavevector: sum and sum of squares over samples of S(q) */
int selm_analysis_structure(selm_analysis* a, double* sum, double* sumsq, long long* samples);
/* per direction: sum and sum of squares over samples of K_d */
int selm_analysis_kinetic(selm_analysis* a, double* sum, double* sumsq, long long* samples);
int selm_analysis_reset(selm_analysis* a);
int selm_analysis_device_bytes(selm_analysis* a, unsigned long long* bytes);
int selm_analysis_destroy(selm_analysis* a);

/* ---- decomposed instance (z slabs over ranks) ----
 * Replaces the reference's MPI slab decomposition of one instance: z slabs
 * with FFTW-MPI transposed layouts (mpi/SELM_Eulerian_Period.cpp:18-51,
 * 348-407) and the summed interpolation (mpi/SELM_Lagrangian_LAMMPS.cpp:102).
 * selm_slab_create makes rank `rank`'s slab of an instance over `nranks`
 * ranks (fused forms, inertial integrator, a grid of 16, 32, 48, 64, 96 or
 * 128 cells per side with nz a multiple of 16 nranks): grid planes
 * [rank nz/nranks, (rank+1) nz/nranks) and a block of the ny (nx/2+1)
 * columns of the half spectrum (selm_slab_layout).  Every rank is given the
 * same monomers and topology and keeps all of them; selm_set_particles,
 * selm_set_topology, selm_initial, selm_get_particles work as for a whole
 * instance.  A step is the four stages below, the same on every rank, with
 * the caller's exchanges between them (buffers from selm_slab_buffers,
 * device pointers, on the slab's stream, sizes in bytes):
 *   selm_slab_gather   -> gather [3][M] (FP32/FP64) holds this slab's part of
 *                         the interpolation; the caller replaces it by the
 *                         sum over the ranks (an all-reduce);
 *   selm_slab_advance  -> work [3][nzl][ny (nx/2+1)] complex: the xy spectrum
 *                         of the slab's planes; the caller's all-to-all
 *                         moves it to cols [3][nz][ncl] of every rank
 *                         (rank r's columns c0..c0+ncl-1, planes in order);
 *   selm_slab_solve    -> cols: the z pass, in place; the caller's
 *                         all-to-all moves the columns back to work;
 *   selm_slab_finish   -> the slab's velocity, the forces at x^{n+1}.
 * selm_slab_velocity reads the slab's velocity [3][nzl][ny][nx].  A slab
 * refuses selm_step and batches. */
int selm_slab_create(const selm_params* params, int rank, int nranks, selm_sim** out);
int selm_slab_layout(const selm_sim* s, int* z0, int* nzl, long long* c0, long long* ncl);
int selm_slab_buffers(selm_sim* s, void** gather, void** work, void** cols, long long* sizes);
int selm_slab_gather(selm_sim* s);
int selm_slab_advance(selm_sim* s);
int selm_slab_solve(selm_sim* s);
int selm_slab_finish(selm_sim* s);
int selm_slab_velocity(selm_sim* s, double* out);

/* kernels this library has launched since it was loaded (all simulations) */
unsigned long long selm_kernel_launches(void);

/* ---- errors ---- */
const char* selm_last_error(void);
const char* selm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SELM_B200_H */
