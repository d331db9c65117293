/*
 * powergrid_b200.h — C ABI of the B200 (sm_100a) implementation of PowerGrid's
 * system-operator path: Gnufft, Gdft, TimeSegmentation, SENSE, pcSenseTimeSeg,
 * QuadPenalty/TVPenalty and solve_pwls_pcg, plus a request server.
 *
 * Plain C: pointers, sizes and status codes only.  Complex vectors are
 * interleaved single-precision pairs (re, im) — the memory layout of
 * std::complex<float> / arma::cx_float.  Image vectors are y-fastest
 * (index = y + Ny*x + Nx*Ny*z, reconSolve.cpp:40-53); coil data are
 * coil-major [coil][sample] (SENSE.cpp:66, 86).
 *
 * Every entry point returns pg_status and never exits the process (the
 * reference prints and calls exit(1), gridding.cpp:454-457; Gnufft.cpp:297-300).
 * pg_last_error() gives a message for the calling thread's last failure.
 *
 * Reference citations are relative to the PowerGrid/ source directory.
 */
#ifndef POWERGRID_B200_H
#define POWERGRID_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pg_status {
  PG_OK = 0,
  PG_INVALID_ARG = 1,
  PG_OUT_OF_MEMORY = 2,
  PG_CUDA_ERROR = 3,
  PG_TIMEOUT = 4,
  PG_CANCELLED = 5,
  PG_NOT_INITIALIZED = 6,
  PG_CUFFT_ERROR = 7,
  PG_REJECTED = 8,     /* admission control: request exceeds the HBM budget */
  PG_NOT_READY = 9     /* pg_poll: request still running */
} pg_status;

/* Opaque handles. */
typedef struct pg_op_s* pg_op;          /* any system operator */
typedef struct pg_server_s* pg_server;  /* request server */

/* ---- library ---------------------------------------------------------- */
/* Select the CUDA device and create the library context.  Calling any other
 * entry point first initialises device 0 implicitly. */
pg_status pg_init(int device);
pg_status pg_shutdown(void);
const char* pg_status_string(pg_status s);
const char* pg_last_error(void);
/* Number of this library's kernel launches since pg_init (instrumentation). */
uint64_t pg_kernel_launch_count(void);

/* ---- operators -------------------------------------------------------- */
/* Gnufft(dataLength, gridos, nx, ny, nz, kx, ky, kz, ix, iy, iz)
 * replaces Gnufft<float>::Gnufft (Gnufft.h:51-53, Gnufft.cpp:34-122).
 * k in cycles/FOV, host arrays of length dataLength (copied).  The image
 * coordinates ix/iy/iz are stored but unused by the math in the reference
 * (Gnufft.cpp:47-49), so they are not taken here.  2-D requires nx == ny
 * (the reference mixes x/y-fastest conventions otherwise: zero_pad2d
 * griddingSupport.cpp:488 vs gridding.cpp:100).  Operator application
 * needs gridos = 2; an operator made with another factor (up to 3.75) serves
 * the spatial interpolation below only, as density compensation uses it. */
pg_status pg_gnufft_create(pg_op* out, uint64_t data_length, float gridos, uint64_t nx, uint64_t ny,
                           uint64_t nz, const float* kx, const float* ky, const float* kz);

/* Gdft(nk, ni, kx, ky, kz, ix, iy, iz, FM_rad_per_s, t_s) replaces
 * Gdft<float>::Gdft (Gdft.h:47-49, Gdft.cpp:33-49). */
pg_status pg_gdft_create(pg_op* out, uint64_t nk, uint64_t ni, const float* kx, const float* ky,
                         const float* kz, const float* ix, const float* iy, const float* iz,
                         const float* field_map, const float* t);

/* GdftR2(nk, ni, kx, ky, kz, ix, iy, iz, FM, t, num_x, num_y, num_z) replaces
 * GdftR2<float>::GdftR2 (GdftR2.h, GdftR2.cpp:32-57): Gdft with each
 * sample-voxel pair weighted by sinc(kx/Nx + Gx t) sinc(ky/Ny + Gy t)
 * sinc(kz/Nz + Gz t), G* the field map's differences (GdftR2.cpp:62-110,
 * ftCpuWithGrads.cpp:93-216).  nx*ny*nz must equal ni. */
pg_status pg_gdftr2_create(pg_op* out, uint64_t nk, uint64_t ni, const float* kx, const float* ky, const float* kz,
                           const float* ix, const float* iy, const float* iz, const float* field_map, const float* t,
                           uint64_t nx, uint64_t ny, uint64_t nz);

/* TimeSegmentation(G, fieldmap, tvec, n1 = data length, n2 = image length, L,
 * interptype, shots) replaces TimeSegmentation<float, Tobj>::TimeSegmentation
 * (TimeSegmentation.h:70-71, TimeSegmentation.cpp:37-221).  G is not owned
 * and must outlive this operator (TimeSegmentation.cpp:53).  interptype 1 =
 * Hanning (TimeSegmentation.cpp:80-93). */
pg_status pg_timeseg_create(pg_op* out, pg_op G, const float* field_map, const float* tvec, uint64_t n1,
                            uint64_t n2, uint64_t L, uint64_t interptype, uint64_t shots);

/* SENSE(G, senseMap (complex, n2*nc, coil-major), n1, n2, nc) replaces
 * SENSE<float, Tobj>::SENSE (SENSE.h:64, SENSE.cpp:33-44).  G not owned. */
pg_status pg_sense_create(pg_op* out, pg_op G, const float* sense_map, uint64_t n1, uint64_t n2, uint64_t nc);

/* pcSenseTimeSeg(kx, ky, kz, nx, ny, nz, nc, t, L, intType, SENSEmap,
 * FieldMap, ShotPhaseMap) replaces pcSenseTimeSeg<float>::pcSenseTimeSeg
 * (pcSenseTimeSeg.h:80-82, pcSenseTimeSeg.cpp:41-125).  nk = total samples
 * (all shots); shots = n_shot_phase / (nx*ny*nz) (pcSenseTimeSeg.cpp:47). */
pg_status pg_pcsense_timeseg_create(pg_op* out, const float* kx, const float* ky, const float* kz, uint64_t nk,
                                    uint64_t nx, uint64_t ny, uint64_t nz, uint64_t nc, const float* t,
                                    uint64_t L, uint64_t interptype, const float* sense_map,
                                    const float* field_map, const float* shot_phase_map, uint64_t n_shot_phase);

/* pcSENSE(kx, ky, kz, nx, ny, nz, nc, t, SENSEmap, FieldMap, ShotPhaseMap)
 * replaces pcSENSE<float>::pcSENSE (pcSENSE.h:76-78, pcSENSE.cpp:40-104):
 * multishot phase-corrected SENSE over one Gdft per shot.  nk = total samples
 * (all shots); shots = n_shot_phase / (nx*ny*nz) (pcSENSE.cpp:44).  Like the
 * reference, both directions weight by exp(+i*ShotPhaseMap) (pcSENSE.cpp:103,
 * 123, 146), so the adjoint is not the exact adjoint of the forward. */
pg_status pg_pcsense_create(pg_op* out, const float* kx, const float* ky, const float* kz, uint64_t nk, uint64_t nx,
                            uint64_t ny, uint64_t nz, uint64_t nc, const float* t, const float* sense_map,
                            const float* field_map, const float* shot_phase_map, uint64_t n_shot_phase);

/* LRobj(NimgSize, N_data, n_rank, n_img, vBasis, All) replaces
 * LRobj<float, Gobj>::LRobj (lowRank/LRobj.h:55, LRobj.cpp:27-35): the
 * partial-separability model x = vec(X), X n_image x rank, whose image i is
 * column i of X * vBasis and goes through ops[i] (operator*, LRobj.cpp:38-50);
 * the adjoint applies ops[i]^H to data column i and multiplies the
 * n_image x n_img stack by vBasis^H (LRobj.cpp:53-66).  v: rank x n_img
 * complex, column-major (interleaved float pairs).  Every ops[i] must be
 * n_data x n_image (a pcSENSE or pcSenseTimeSeg plan, or any operator of
 * that shape); they are borrowed and must outlive the model, as the
 * reference holds raw pointers.  The model is (n_data*n_img) x
 * (n_image*rank). */
pg_status pg_lowrank_create(pg_op* out, uint64_t n_image, uint64_t n_data, uint64_t rank, uint64_t n_img,
                            const float* v, const pg_op* ops);

pg_status pg_op_destroy(pg_op op);
/* Lengths of the data vector (operator* output) and image vector. */
pg_status pg_op_shape(pg_op op, uint64_t* n_data, uint64_t* n_image);

/* operator* (forward) and operator/ (adjoint) on HOST buffers: the
 * Col<complex<float>> interface of every operator above (e.g.
 * Gnufft.cpp:153-211, SENSE.cpp:51-97).  Synchronous. */
pg_status pg_op_forward(pg_op op, const float* x, float* y);
pg_status pg_op_adjoint(pg_op op, const float* y, float* x);

/* The same on DEVICE buffers, stream-ordered (stream may be NULL = the
 * library's default stream).  No host synchronisation. */
pg_status pg_op_forward_device(pg_op op, const void* x_dev, void* y_dev, void* stream);
pg_status pg_op_adjoint_device(pg_op op, const void* y_dev, void* x_dev, void* stream);

/* ---- interpolation without the FFT, and the direct reconstruction -------- */
/* Cells of the operator's oversampled grid (Gnufft.cpp:56-61). */
pg_status pg_gnufft_grid_length(pg_op G, uint64_t* n_cells);
/* Gnufft::forwardSpatialInterp (Gnufft.cpp:213-258): grid (complex, n_cells,
 * the reference's unshifted y-fastest layout, gridding.cpp:66) -> samples
 * (complex, data_length).  Host buffers, synchronous. */
pg_status pg_gnufft_forward_spatial_interp(pg_op G, const float* grid, float* samples);
/* Gnufft::adjointSpatialInterp (Gnufft.cpp:261-330): samples -> grid (every
 * cell written). */
pg_status pg_gnufft_adjoint_spatial_interp(pg_op G, const float* samples, float* grid);
/* The same on device buffers, stream-ordered. */
pg_status pg_gnufft_forward_spatial_interp_device(pg_op G, const void* grid_dev, void* samples_dev, void* stream);
pg_status pg_gnufft_adjoint_spatial_interp_device(pg_op G, const void* samples_dev, void* grid_dev, void* stream);
/* calc3DDensityCompensation(kx, ky, kz, Ninplane, Nz)
 * (reconSupport/directRecon.cpp:28-61): two Pipe iterations on a 3x
 * oversampled grid, normalised to unit L2 norm; dcf = n floats. */
pg_status pg_density_compensation(const float* kx, const float* ky, const float* kz, uint64_t n,
                                  uint64_t n_inplane, uint64_t nz, float* dcf);
/* The per-coil step of gridCoilImages (directRecon.cpp:108-133):
 * images[c] = G / (dcf .* data[c]) for nc coils; data coil-major [c][sample],
 * images coil-major [c][voxel] (complex). */
pg_status pg_grid_coil_images(pg_op G, const float* dcf, const float* data, uint64_t nc, float* images);
/* calcSumOfSquaresImage (directRecon.cpp:63-73): out[p] = sqrt(sum_c |img_c[p]|)
 * (a sum of magnitudes, as the reference computes it). */
pg_status pg_sum_of_squares_image(const float* coil_images, uint64_t n, uint64_t nc, float* out);

/* y = Gdft * x for one coil, computed without allocating any device memory.
 * No counterpart in the reference: it exists for callers that manage all
 * device memory themselves (their own pool or a fixed budget) or that must
 * not meet cudaMalloc's implicit synchronisation or an allocation failure
 * mid-run.  Every pointer is a DEVICE pointer owned by the caller: the
 * operator's inputs as for pg_gdft_create (nk samples, ni voxels), x (ni
 * complex) and y (nk complex).  Scratch lives in a fixed 4 MiB device array
 * held by every GPU that loads the library until exit, so nk is limited to
 * 524288 samples (larger sizes return PG_INVALID_ARG).  The array is shared
 * by all calls: calls whose work overlaps on the GPU race and must be
 * ordered by the caller.  The call runs on the device given to pg_init (the
 * library makes it current), so the buffers must live on that device.  The
 * first call after pg_init looks up the array's device address; make that
 * first call before any stream capture.
 * Stream-ordered on `stream` (NULL = the library's stream). */
pg_status pg_gdft_forward_noalloc(uint64_t nk, uint64_t ni, const float* kx, const float* ky, const float* kz,
                                  const float* ix, const float* iy, const float* iz, const float* field_map,
                                  const float* t, const void* x_dev, void* y_dev, void* stream);

/* ---- regularizers and solver ----------------------------------------- */
typedef enum pg_penalty_kind { PG_PENALTY_QUAD = 0, PG_PENALTY_TV = 1 } pg_penalty_kind;

/* QuadPenalty(nx, ny, nz, beta, dims2penalize) (QuadPenalty.h:43) and
 * TVPenalty(nx, ny, nz, beta, delta, dims2penalize) (TVPenalty.h:42). */
typedef struct pg_penalty {
  int kind;                 /* pg_penalty_kind */
  uint64_t nx, ny, nz;
  float beta;
  float delta;              /* TV only */
  uint64_t dims2penalize;   /* 2 or 3; reference default 3 */
} pg_penalty;

/* solve_pwls_pcg(xInitial, A, W, yi, R, niter) (solve_pwls_pcg.hpp:48-51).
 * Host buffers.  x0 may be NULL (zeros, as reconSolve.h:75-76); W may be
 * NULL (ones, reconSolve.h:73-74).  Inner products, step sizes and the CG
 * coefficient are accumulated in FP64 on the device; each iteration runs as
 * one CUDA graph.  iters_done (may be NULL) receives the number of
 * completed iterations (early exits as solve_pwls_pcg.hpp:88-91, 113-116,
 * 137-145). */
pg_status pg_pcg_solve(pg_op A, const float* x0, const float* W, const float* y, const pg_penalty* R,
                       uint64_t niter, float* x_out, uint64_t* iters_done);

/* The same on device buffers, stream-ordered; iters_done_dev (may be NULL)
 * is a device uint32. */
pg_status pg_pcg_solve_device(pg_op A, const void* x0_dev, const void* W_dev, const void* y_dev,
                              const pg_penalty* R, uint64_t niter, void* x_out_dev, void* iters_done_dev,
                              void* stream);

/* Checkpoint / resume of a solve (no counterpart in the reference, which
 * keeps no state between calls).  The state the solver holds on the
 * operator between iterations — x, Ax, the residual, the search direction
 * (and the previous one for a QuadPenalty), the FP64 scalars and the
 * iteration counters — is copied to a host blob of pg_pcg_state_size bytes
 * after a solve (or a cancelled one: cancellation stops between
 * iterations), and loaded onto an operator of the same shape, e.g. a new
 * plan on another GPU.  pg_pcg_resume then runs niter more iterations from
 * it, exactly as the uninterrupted solve would continue; iters_done counts
 * from the original start.  The blob records the operator shape and the
 * penalty (kind, size, beta, delta, dims2penalize) it was computed for;
 * pg_pcg_state_load and pg_pcg_resume refuse another one with
 * PG_INVALID_ARG. */
pg_status pg_pcg_state_size(pg_op A, uint64_t* bytes);
pg_status pg_pcg_state_save(pg_op A, void* host, uint64_t bytes);
pg_status pg_pcg_state_load(pg_op A, const pg_penalty* R, const void* host, uint64_t bytes);
pg_status pg_pcg_resume(pg_op A, const float* W, const float* y, const pg_penalty* R, uint64_t niter, float* x_out,
                        uint64_t* iters_done);
pg_status pg_pcg_resume_device(pg_op A, const void* W_dev, const void* y_dev, const pg_penalty* R, uint64_t niter,
                               void* x_out_dev, void* iters_done_dev, void* stream);

/* reconSolve(data, Sg, R, kx, ky, kz, Nx, Ny, Nz, tvec, niter)
 * (reconSolve.h:63-82): W = 1, x0 = 0. */
pg_status pg_recon_solve(pg_op Sg, const pg_penalty* R, const float* data, uint64_t niter, float* image_out);

/* Penalty pieces (Robject.cpp:143-193) on device buffers, for tests. */
pg_status pg_penalty_gradient_device(const pg_penalty* R, const void* x_dev, void* g_dev, void* stream);
pg_status pg_penalty_denom_device(const pg_penalty* R, const void* ddir_dev, const void* x_dev, double* out_host);

/* solve_pwls_pcg(xInitial, A, W, yi, R_lr, niter) with
 * R_lr = R_lowRank(R, rank, nImages, vBasis) (lowRank/R_lowRank.h:52,
 * R_lowRank.cpp:27-95; composed so in lowRank/oscillateRecon.cpp:256-265):
 * R (nx*ny*nz = the model's image length) applied to the columns of
 * X * vBasis^H.  As in the reference, the wrapper's gradient is
 * vectorise(strans(vBasis) * strans(Y)) -- stored rank-fastest -- which is
 * defined only when rank == n_img (PG_INVALID_ARG otherwise), and its Denom
 * is beta * sum_i R.Denom(...), R.Denom already carrying beta.  v: rank x
 * n_img complex, column-major.  The step scalars are FP64 on the host (one
 * synchronisation per inner product).  Host buffers. */
pg_status pg_pcg_solve_lowrank(pg_op A, const float* x0, const float* W, const float* y, const pg_penalty* R,
                               uint64_t rank, uint64_t n_img, const float* v, uint64_t niter, float* x_out,
                               uint64_t* iters_done);
/* The same on device buffers (v stays a host array); returns after the
 * solve (iters_done is a host pointer, may be NULL). */
pg_status pg_pcg_solve_lowrank_device(pg_op A, const void* x0_dev, const void* W_dev, const void* y_dev,
                                      const pg_penalty* R, uint64_t rank, uint64_t n_img, const float* v,
                                      uint64_t niter, void* x_out_dev, uint64_t* iters_done, void* stream);
/* R_lowRank::Gradient and ::Denom (R_lowRank.cpp:50-87) on device buffers, for tests. */
pg_status pg_lowrank_penalty_gradient_device(const pg_penalty* R, uint64_t rank, uint64_t n_img, const float* v,
                                             const void* x_dev, void* g_dev, void* stream);
pg_status pg_lowrank_penalty_denom_device(const pg_penalty* R, uint64_t rank, uint64_t n_img, const float* v,
                                          const void* ddir_dev, const void* x_dev, double* out_host);

/* ---- ingest and output formats ---------------------------------------- */
/* One acquisition as ISMRMRD::Acquisition presents it: the encoding counters
 * the reference sorts by (acqTracking.cpp:64-75), the sample and channel
 * counts, the samples channel-major (acq.data(sample, channel) =
 * data[2*(channel*number_of_samples + sample)], complex) and the trajectory
 * sample-major with kx, ky, kz, t as its first four rows (acq.traj(dim,
 * sample) = traj[sample*trajectory_dimensions + dim]).  The arrays are
 * borrowed by the index built over them. */
typedef struct pg_acquisition {
  uint32_t kspace_encode_step_1;   /* shot */
  uint32_t kspace_encode_step_2;   /* partition */
  uint32_t slice, repetition, average, contrast, phase;
  uint32_t number_of_samples;
  uint32_t active_channels;
  uint32_t trajectory_dimensions;  /* >= 4 */
  const float* data;
  const float* traj;
} pg_acquisition;

/* encodingLimits.<counter>.maximum + 1 for each counter (acqTracking.cpp:17-26). */
typedef struct pg_encoding_limits {
  uint32_t shots, partitions, slices, repetitions, averages, contrasts, phases;
} pg_encoding_limits;

typedef struct pg_acq_index_s* pg_acq_index;

/* acqTracking(d, hdr) (acqTracking.h:14, acqTracking.cpp:9-76): the table
 * (shot, partition, slice, repetition, average, contrast, phase) ->
 * acquisition number, -1 where none; a later acquisition with the same
 * counters replaces an earlier one. */
pg_status pg_acq_index_create(pg_acq_index* out, const pg_acquisition* acqs, uint64_t n_acq,
                              const pg_encoding_limits* limits);
pg_status pg_acq_index_destroy(pg_acq_index ix);
/* acqArray(NShot, NPar, NSlice, NRep, NAvg, NEcho, NPhase) (acqTracking.cpp:73). */
pg_status pg_acq_index_lookup(pg_acq_index ix, uint32_t shot, uint32_t partition, uint32_t slice, uint32_t repetition,
                              uint32_t average, uint32_t contrast, uint32_t phase, int64_t* acq);
/* The encoding limits the index was built with. */
pg_status pg_acq_index_limits(pg_acq_index ix, pg_encoding_limits* limits);
/* getCompleteISMRMRDAcqData(d, acqTrack, NSlice, NRep, NAve, NEcho, NPhase,
 * data, kx, ky, kz, tvec) (processIsmrmrd.hpp:361-471): the sizes first
 * (acquisitions found, samples and channels of each; all must match), then
 * the arrays: data complex n_channels x n_acq x n_samples (coil-major, the
 * reference's permute + vectorise), kx/ky/kz/t n_acq x n_samples, the
 * acquisitions in partition-major, shot-minor order.  Host buffers. */
pg_status pg_acq_gather_size(pg_acq_index ix, uint32_t slice, uint32_t repetition, uint32_t average,
                             uint32_t contrast, uint32_t phase, uint64_t* n_acq, uint64_t* n_samples,
                             uint64_t* n_channels);
pg_status pg_acq_gather(pg_acq_index ix, uint32_t slice, uint32_t repetition, uint32_t average, uint32_t contrast,
                        uint32_t phase, float* data, float* kx, float* ky, float* kz, float* t);
/* The same into DEVICE buffers: each acquisition's block is copied to the
 * device once and the coil-major permutation runs on the GPU.  Stream-
 * ordered; the host arrays must stay valid until the stream reaches the
 * copies. */
pg_status pg_acq_gather_device(pg_acq_index ix, uint32_t slice, uint32_t repetition, uint32_t average,
                               uint32_t contrast, uint32_t phase, void* data_dev, void* kx_dev, void* ky_dev,
                               void* kz_dev, void* t_dev, void* stream);

/* writeNiftiRealImage(filename, imageData, Nx, Ny, Nz, Nslab, N_TR)
 * (processNIFTI.hpp:37-99): "<filename>.nii", a NIfTI-1 header (dim[0] = 3,
 * float32, vox_offset 352, scl_slope 100, mm units, magic "n+1"), a zero
 * 4-byte extender and the voxels in the vector's own order.  Header fields
 * the reference leaves unset are zero. */
pg_status pg_write_nifti_real(const char* filename, const float* image, uint64_t nx, uint64_t ny, uint64_t nz,
                              uint64_t nslab, uint64_t ntr);
/* writeNiftiMagPhsImage (processNIFTI.hpp:103-117): "<filename>_mag.nii" and
 * "<filename>_phs.nii" from a complex image (abs and arg in float). */
pg_status pg_write_nifti_mag_phs(const char* filename, const float* image, uint64_t nx, uint64_t ny, uint64_t nz,
                                 uint64_t nslab, uint64_t ntr);

/* ---- request server (continuous batching) ---------------------------- */
typedef struct pg_server_config {
  uint64_t hbm_budget_bytes;   /* admission limit on the summed footprint of resident jobs */
  uint32_t max_inflight;       /* jobs on the GPU at once: one worker thread and stream each */
  uint32_t reserved;           /* must be 0 */
} pg_server_config;

/* A time-segmented SENSE reconstruction request:
 * SENSE<TimeSegmentation<Gnufft>> + QuadPenalty with reconSolve semantics
 * (reconSolve.h:63-82), for n_slices independent images that share one
 * trajectory (the slice loop of PowerGridIsmrmrd.cpp:191-264).  The slices
 * are batched: a job is all of the request's slices (or as many as fit the
 * HBM budget) solved as one stacked operator whose gridding launches carry
 * every slice's coils, with one PCG that keeps its inner products, step sizes
 * and early exits per slice, so each slice's image is that of its own solve.
 * Arrays (host memory, valid until completion):
 *   kx, ky, kz, t   n_samples                  (k in cycles/FOV, t in s)
 *   field_map       n_slices * nx*ny*nz        (rad/s)
 *   sense_map       n_slices * nx*ny*nz*nc     (complex, coil-major per slice)
 *   data            n_slices * n_samples*nc    (complex, coil-major per slice)
 *   image_out       n_slices * nx*ny*nz        (complex, written on completion) */
typedef struct pg_request {
  uint64_t nx, ny, nz, n_slices, nc, n_samples, L, niter;
  float beta;
  const float* kx; const float* ky; const float* kz; const float* t;
  const float* field_map;
  const float* sense_map;
  const float* data;
  float* image_out;
} pg_request;

typedef struct pg_request_stats {
  double t_submit_ms, t_start_ms, t_done_ms;   /* host steady clock; start = first job admitted */
  uint64_t iters_done;                         /* PCG iterations completed, all slices */
  uint64_t bytes_resident;                     /* admission footprint of one slice */
  pg_status status;
  double setup_ms;                             /* summed over jobs: operator construction */
  double solve_ms;                             /* summed over jobs: PCG solve and image copy-out */
  uint64_t jobs;                               /* jobs the request was split into (batches of slices) */
  char error[160];                             /* the first failed job's message, or empty */
} pg_request_stats;

pg_status pg_server_create(pg_server* out, const pg_server_config* cfg);
pg_status pg_server_destroy(pg_server s);
/* Request buffers must stay valid until pg_poll reports completion. */
pg_status pg_submit(pg_server s, const pg_request* req, uint64_t* ticket);
/* PG_OK when done (stats filled), PG_NOT_READY while queued/running. */
pg_status pg_poll(pg_server s, uint64_t ticket, pg_request_stats* stats);
pg_status pg_wait(pg_server s, uint64_t ticket, pg_request_stats* stats);
pg_status pg_cancel(pg_server s, uint64_t ticket);
/* Device bytes one slice job of the request holds while resident (the
 * admission metric; an upper bound of what the job allocates). */
uint64_t pg_request_footprint(const pg_request* req);

/* The reference ISMRMRD driver's image loop as one request
 * (PowerGridIsmrmrd.cpp:191-264): every image of the acquisition index, in
 * its loop order (slice outermost, then phase, contrast, average, and
 * repetition innermost: image k = (((slice * phases + phase) * contrasts +
 * contrast) * averages + average) * repetitions + repetition), each gathered
 * as getCompleteISMRMRDAcqData does (pg_acq_gather), with its slice's field
 * map and coil maps (getISMRMRDCompleteFieldMap / getISMRMRDCompleteSENSEMap,
 * processIsmrmrd.hpp:196-266), reconstructed as
 * SENSE<TimeSegmentation<Gnufft>> (Hanning interpolation, one shot) +
 * QuadPenalty(beta, 3 dimensions) with reconSolve.  Images whose gathered
 * trajectories are identical are batched as the slices of pg_submit are.
 * The gather runs in pg_submit_acquisitions, so the acquisitions may be
 * released on return; the maps and image_out must stay valid until
 * completion.  Every image needs at least one acquisition and all the same
 * channel count (the coil maps are sized by it); otherwise PG_INVALID_ARG. */
typedef struct pg_acq_request {
  uint64_t nx, ny, nz;
  uint64_t L;               /* time segments; 0 = ceil((max t - min t) / 2 ms), the driver's default */
  uint64_t niter;
  float beta;
  const float* field_map;   /* slices * nx*ny*nz (rad/s), slice-major */
  const float* sense_map;   /* slices * nx*ny*nz*nc (complex, coil-major per slice) */
  float* image_out;         /* images * nx*ny*nz (complex) */
} pg_acq_request;
pg_status pg_submit_acquisitions(pg_server s, pg_acq_index ix, const pg_acq_request* req, uint64_t* ticket);

/* ---- device-side index checks ------------------------------------------ */
/* In the PG_CHECKS build (libpowergrid_b200_checks.so, build(checks=True))
 * the gridding kernels check every index they derive from the sample binning
 * (window start inside the tile, sample count within the staging area,
 * permutation entry inside the data) and record the first failed check
 * instead of making the access: *record = (site << 48) | (low 48 bits of the
 * offending value), sites 1 spread sample count, 2 / 3 spread window start
 * (3-D or generic / 2-D), 4 spread permutation entry, 5 gather window start,
 * 6 gather permutation entry; 0 if no check failed since the last call.
 * Reading clears the record and synchronises the device.  *enabled = 1 in
 * the checks build; the product build has no checks (*enabled = 0, *record =
 * 0). */
pg_status pg_checks_read(uint64_t* record, int* enabled);

/* ---- instrumentation and fault injection (host-side only) ------------ */
/* Stage timing: while enabled, the NUFFT and Gdft pipelines record a CUDA
 * event pair around each stage kernel on the stream they run on (also inside
 * captured CUDA graphs).  pg_profile_stage_ms returns the elapsed time of the
 * most recent recorded pair of a stage ("pre", "fft_fwd", "gather", "prep",
 * "spread", "fft_adj", "post", "dft_fwd", "dft_adj"); the caller must have
 * synchronised the stream.  Returns PG_NOT_READY if the stage never ran. */
pg_status pg_profile_enable(int on);
pg_status pg_profile_stage_ms(const char* stage, float* ms);
/* Restrict recording to one stage (NULL or "" = every stage), so that a timed
 * run carries only the event pair it needs. */
pg_status pg_profile_only(const char* stage);

/* Make the n-th device allocation from now fail with PG_OUT_OF_MEMORY
 * (n = 0 disables). */
void pg_debug_fail_allocation_after(uint64_t n);
/* Kaiser-Bessel lookup table as built by Gnufft (griddingSupport.cpp:52-76;
 * beta from Gnufft.cpp:84-88).  Returns its length. */
uint64_t pg_util_kb_lut(float gridos, float* lut_out, uint64_t cap, float* beta_out);
/* The adjoint's sample binning for a Gnufft operator: per-sample bin key in
 * original order, and the stable sorted permutation. */
pg_status pg_util_gnufft_binning(pg_op G, uint32_t* keys_out, uint32_t* perm_out, uint64_t* n_bins_out);

#ifdef __cplusplus
}
#endif
#endif /* POWERGRID_B200_H */
