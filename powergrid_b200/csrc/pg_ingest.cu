// Ingest and output formats around the reconstruction (the reference reads
// ISMRMRD/HDF5 files and writes NIfTI images; the HDF5 layer is replaced by
// an in-memory acquisition list, the NIfTI writer is kept byte for byte).
//
//   acquisition index   acqTracking::acqTracking (acqTracking.cpp:9-76): a
//                       7-D table (shot, partition, slice, repetition,
//                       average, contrast, phase) -> acquisition number, -1
//                       where none; a later acquisition with the same
//                       counters replaces an earlier one (:73).
//   per-image gather    getCompleteISMRMRDAcqData (processIsmrmrd.hpp:361-471):
//                       for one (slice, repetition, average, contrast, phase),
//                       the acquisitions in partition-major, shot-minor order
//                       (:380-381, :406-407); data (nro x nc x nacq) permuted to
//                       (nro x nacq x nc) and vectorised (:455-458), so coil c's
//                       samples of acquisition a start at (c*nacq + a)*nro;
//                       traj rows 0-3 are kx, ky, kz, t (:444-448), [a][sample].
//   NIfTI writer        writeNiftiRealImage / writeNiftiMagPhsImage
//                       (processNIFTI.hpp:37-117): a 348-byte NIfTI-1 header,
//                       a 4-byte zero extender, float32 voxels in the image
//                       vector's own order.
//
// The device gather uploads each acquisition's contiguous block once (one
// copy per acquisition, no host repacking) and permutes on the GPU.
#include <algorithm>
#include <cmath>
#include <complex>
#include <memory>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pg_common.cuh"

struct pg_acq_index_s {
  std::vector<pg_acquisition> acqs;     // borrowed sample and trajectory pointers
  pg_encoding_limits lim{};
  std::vector<int64_t> table;           // shot fastest, phase slowest
  pg::DevBuf<float2> stage;             // device gather: acquisitions as uploaded
  pg::DevBuf<float> stage_traj;
  uint64_t at(uint32_t shot, uint32_t par, uint32_t slice, uint32_t rep, uint32_t avg, uint32_t echo,
              uint32_t phase) const {
    return shot + (uint64_t)lim.shots *
                      (par + (uint64_t)lim.partitions *
                                 (slice + (uint64_t)lim.slices *
                                              (rep + (uint64_t)lim.repetitions *
                                                         (avg + (uint64_t)lim.averages *
                                                                    (echo + (uint64_t)lim.contrasts * phase)))));
  }
};

namespace pg {
namespace {

bool counters_inside(const pg_encoding_limits& l, uint32_t shot, uint32_t par, uint32_t slice, uint32_t rep,
                     uint32_t avg, uint32_t echo, uint32_t phase) {
  return shot < l.shots && par < l.partitions && slice < l.slices && rep < l.repetitions && avg < l.averages &&
         echo < l.contrasts && phase < l.phases;
}

// The acquisitions of one image in the reference's order (partition outer,
// shot inner), with their common sample and channel counts.
pg_status select(const pg_acq_index_s& ix, uint32_t slice, uint32_t rep, uint32_t avg, uint32_t echo,
                 uint32_t phase, std::vector<int64_t>* sel, uint32_t* nro, uint32_t* nc) {
  if (!counters_inside(ix.lim, 0, 0, slice, rep, avg, echo, phase))
    return set_error(PG_INVALID_ARG, "acquisition gather: counters outside the encoding limits");
  sel->clear();
  *nro = 0;
  *nc = 0;
  for (uint32_t par = 0; par < ix.lim.partitions; ++par)
    for (uint32_t shot = 0; shot < ix.lim.shots; ++shot) {
      const int64_t a = ix.table[ix.at(shot, par, slice, rep, avg, echo, phase)];
      if (a < 0) continue;
      const pg_acquisition& q = ix.acqs[(size_t)a];
      if (sel->empty()) {
        *nro = q.number_of_samples;
        *nc = q.active_channels;
      } else if (q.number_of_samples != *nro || q.active_channels != *nc) {
        // the reference sizes its work arrays from the first acquisition
        // (:386-397) and cannot hold a different one
        return set_error(PG_INVALID_ARG, "acquisition %lld has %u samples x %u channels, the image's first %u x %u",
                         (long long)a, q.number_of_samples, q.active_channels, *nro, *nc);
      }
      sel->push_back(a);
    }
  return PG_OK;
}

// out[(c*nacq + a)*nro + s] = stage[(a*nc + c)*nro + s]; traj rows split per
// sample (trajectory_dimensions = td): kx/ky/kz/t[a*nro + s].
__global__ void k_acq_permute(uint64_t nro, uint32_t nc, uint64_t nacq, const float2* __restrict__ stage,
                              const float* __restrict__ traj, uint32_t td, float2* __restrict__ data,
                              float* __restrict__ kx, float* __restrict__ ky, float* __restrict__ kz,
                              float* __restrict__ t) {
  const uint64_t total = nro * nc * nacq;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t s = i % nro;
    const uint64_t ca = i / nro;
    const uint64_t a = ca % nacq, c = ca / nacq;
    data[i] = stage[(a * nc + c) * nro + s];
    if (c == 0) {
      const float* r = traj + (a * nro + s) * td;
      const uint64_t o = a * nro + s;
      kx[o] = r[0];
      ky[o] = r[1];
      kz[o] = r[2];
      t[o] = r[3];
    }
  }
}

// NIfTI-1 header (processNIFTI.hpp:44-86) at the standard's byte offsets.
// Fields the reference leaves uninitialised are written as zero.
void nifti_header(unsigned char (&h)[348], uint64_t nx, uint64_t ny, uint64_t nz, uint64_t nslab, uint64_t ntr) {
  std::memset(h, 0, sizeof(h));
  auto i32 = [&](int off, int32_t v) { std::memcpy(h + off, &v, 4); };
  auto i16 = [&](int off, int16_t v) { std::memcpy(h + off, &v, 2); };
  auto f32 = [&](int off, float v) { std::memcpy(h + off, &v, 4); };
  i32(0, 348);                                  // sizeof_hdr = MIN_HEADER_SIZE
  const int16_t dim[8] = {3, (int16_t)nx, (int16_t)ny, (int16_t)nz, (int16_t)nslab, (int16_t)ntr, 1, 1};
  for (int k = 0; k < 8; ++k) i16(40 + 2 * k, dim[k]);
  i16(70, 16);                                  // datatype NIFTI_TYPE_FLOAT32
  i16(72, 32);                                  // bitpix
  for (int k = 0; k < 4; ++k) f32(76 + 4 * k, 1.0f);   // pixdim[0..3]
  f32(108, 352.0f);                             // vox_offset = NII_HEADER_SIZE
  f32(112, 100.0f);                             // scl_slope
  h[123] = 2;                                   // xyzt_units NIFTI_UNITS_MM
  std::memcpy(h + 344, "n+1\0", 4);             // magic
}

pg_status nifti_write(const std::string& path, const float* vox, uint64_t n, uint64_t nx, uint64_t ny, uint64_t nz,
                      uint64_t nslab, uint64_t ntr) {
  unsigned char h[348];
  nifti_header(h, nx, ny, nz, nslab, ntr);
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return set_error(PG_INVALID_ARG, "NIfTI: cannot open %s for writing", path.c_str());
  const unsigned char pad[4] = {0, 0, 0, 0};
  const bool ok = std::fwrite(h, 1, 348, f) == 348 && std::fwrite(pad, 1, 4, f) == 4 &&
                  std::fwrite(vox, sizeof(float), n, f) == n;
  const bool closed = std::fclose(f) == 0;
  if (!ok || !closed) return set_error(PG_INVALID_ARG, "NIfTI: short write to %s", path.c_str());
  return PG_OK;
}

pg_status nifti_dims(uint64_t nx, uint64_t ny, uint64_t nz, uint64_t nslab, uint64_t ntr, uint64_t* n) {
  const uint64_t d[5] = {nx, ny, nz, nslab, ntr};
  uint64_t p = 1;
  for (uint64_t v : d) {
    if (v == 0 || v > 32767) return set_error(PG_INVALID_ARG, "NIfTI: dimension %llu outside 1..32767",
                                              (unsigned long long)v);
    p *= v;
  }
  *n = p;
  return PG_OK;
}

}  // namespace
}  // namespace pg

using namespace pg;

extern "C" {

pg_status pg_acq_index_create(pg_acq_index* out, const pg_acquisition* acqs, uint64_t n_acq,
                              const pg_encoding_limits* limits) {
  if (!out || !limits || (n_acq && !acqs)) return set_error(PG_INVALID_ARG, "acquisition index: null argument");
  const pg_encoding_limits& l = *limits;
  const uint64_t cells = (uint64_t)l.shots * l.partitions * l.slices * l.repetitions * l.averages * l.contrasts *
                         l.phases;
  if (cells == 0) return set_error(PG_INVALID_ARG, "acquisition index: an encoding limit is zero");
  if (cells > (1ull << 28)) return set_error(PG_INVALID_ARG, "acquisition index: %llu cells", (unsigned long long)cells);
  auto ix = std::make_unique<pg_acq_index_s>();
  ix->lim = l;
  ix->table.assign(cells, -1);   // acqTracking.cpp:52 (-1 = no acquisition)
  ix->acqs.assign(acqs, acqs + n_acq);
  for (uint64_t a = 0; a < n_acq; ++a) {
    const pg_acquisition& q = acqs[a];
    if (!counters_inside(l, q.kspace_encode_step_1, q.kspace_encode_step_2, q.slice, q.repetition, q.average,
                         q.contrast, q.phase))
      return set_error(PG_INVALID_ARG, "acquisition %llu: counters outside the encoding limits",
                       (unsigned long long)a);
    if (!q.data || !q.traj || q.number_of_samples == 0 || q.active_channels == 0 || q.trajectory_dimensions < 4)
      return set_error(PG_INVALID_ARG, "acquisition %llu: no samples, channels or 4-D trajectory",
                       (unsigned long long)a);
    ix->table[ix->at(q.kspace_encode_step_1, q.kspace_encode_step_2, q.slice, q.repetition, q.average, q.contrast,
                     q.phase)] = (int64_t)a;   // acqTracking.cpp:73
  }
  *out = ix.release();
  return PG_OK;
}

pg_status pg_acq_index_destroy(pg_acq_index ix) {
  if (!ix) return PG_OK;
  if (ix->stage.p || ix->stage_traj.p) cudaDeviceSynchronize();
  delete ix;
  return PG_OK;
}

pg_status pg_acq_index_lookup(pg_acq_index ix, uint32_t shot, uint32_t partition, uint32_t slice, uint32_t repetition,
                              uint32_t average, uint32_t contrast, uint32_t phase, int64_t* acq) {
  if (!ix || !acq) return set_error(PG_INVALID_ARG, "acquisition index: null argument");
  if (!counters_inside(ix->lim, shot, partition, slice, repetition, average, contrast, phase))
    return set_error(PG_INVALID_ARG, "acquisition index: counters outside the encoding limits");
  *acq = ix->table[ix->at(shot, partition, slice, repetition, average, contrast, phase)];
  return PG_OK;
}

pg_status pg_acq_index_limits(pg_acq_index ix, pg_encoding_limits* limits) {
  if (!ix || !limits) return set_error(PG_INVALID_ARG, "acquisition index: null argument");
  *limits = ix->lim;
  return PG_OK;
}

pg_status pg_acq_gather_size(pg_acq_index ix, uint32_t slice, uint32_t repetition, uint32_t average,
                             uint32_t contrast, uint32_t phase, uint64_t* n_acq, uint64_t* n_samples,
                             uint64_t* n_channels) {
  if (!ix || !n_acq || !n_samples || !n_channels) return set_error(PG_INVALID_ARG, "acquisition gather: null argument");
  std::vector<int64_t> sel;
  uint32_t nro = 0, nc = 0;
  PG_TRY(select(*ix, slice, repetition, average, contrast, phase, &sel, &nro, &nc));
  *n_acq = sel.size();
  *n_samples = nro;
  *n_channels = nc;
  return PG_OK;
}

pg_status pg_acq_gather(pg_acq_index ix, uint32_t slice, uint32_t repetition, uint32_t average, uint32_t contrast,
                        uint32_t phase, float* data, float* kx, float* ky, float* kz, float* t) {
  if (!ix || !data || !kx || !ky || !kz || !t) return set_error(PG_INVALID_ARG, "acquisition gather: null argument");
  std::vector<int64_t> sel;
  uint32_t nro = 0, nc = 0;
  PG_TRY(select(*ix, slice, repetition, average, contrast, phase, &sel, &nro, &nc));
  const uint64_t na = sel.size();
  for (uint64_t a = 0; a < na; ++a) {
    const pg_acquisition& q = ix->acqs[(size_t)sel[a]];
    for (uint32_t c = 0; c < nc; ++c)
      std::memcpy(data + 2 * ((c * na + a) * nro), q.data + 2 * ((uint64_t)c * nro), nro * 2 * sizeof(float));
    for (uint32_t s = 0; s < nro; ++s) {
      const float* r = q.traj + (uint64_t)s * q.trajectory_dimensions;
      kx[a * nro + s] = r[0];
      ky[a * nro + s] = r[1];
      kz[a * nro + s] = r[2];
      t[a * nro + s] = r[3];
    }
  }
  return PG_OK;
}

pg_status pg_acq_gather_device(pg_acq_index ix, uint32_t slice, uint32_t repetition, uint32_t average,
                               uint32_t contrast, uint32_t phase, void* data_dev, void* kx_dev, void* ky_dev,
                               void* kz_dev, void* t_dev, void* stream) {
  if (!ix || !data_dev || !kx_dev || !ky_dev || !kz_dev || !t_dev)
    return set_error(PG_INVALID_ARG, "acquisition gather: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  std::vector<int64_t> sel;
  uint32_t nro = 0, nc = 0;
  PG_TRY(select(*ix, slice, repetition, average, contrast, phase, &sel, &nro, &nc));
  const uint64_t na = sel.size();
  if (na == 0) return PG_OK;
  uint32_t td = 0;
  for (int64_t a : sel) td = std::max(td, ix->acqs[(size_t)a].trajectory_dimensions);
  const uint64_t block = (uint64_t)nro * nc;
  // earlier gathers on another stream may still read the staging buffers
  if (ix->stage.p) PG_CUDA(cudaDeviceSynchronize());
  PG_TRY(ix->stage.alloc(block * na));
  PG_TRY(ix->stage_traj.alloc((uint64_t)nro * td * na));
  for (uint64_t a = 0; a < na; ++a) {
    const pg_acquisition& q = ix->acqs[(size_t)sel[a]];
    PG_CUDA(cudaMemcpyAsync(ix->stage.p + a * block, q.data, block * sizeof(float2), cudaMemcpyHostToDevice, s));
    if (q.trajectory_dimensions == td) {
      PG_CUDA(cudaMemcpyAsync(ix->stage_traj.p + a * (uint64_t)nro * td, q.traj, (uint64_t)nro * td * sizeof(float),
                              cudaMemcpyHostToDevice, s));
    } else {
      PG_CUDA(cudaMemcpy2DAsync(ix->stage_traj.p + a * (uint64_t)nro * td, td * sizeof(float), q.traj,
                                q.trajectory_dimensions * sizeof(float), q.trajectory_dimensions * sizeof(float), nro,
                                cudaMemcpyHostToDevice, s));
    }
  }
  const uint64_t total = block * na;
  const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(total, 256), 8ull * sm_count());
  PG_LAUNCH(k_acq_permute, grid, 256, 0, s, (uint64_t)nro, nc, na, ix->stage.p, ix->stage_traj.p, td,
            (float2*)data_dev, (float*)kx_dev, (float*)ky_dev, (float*)kz_dev, (float*)t_dev);
  return PG_OK;
}

pg_status pg_write_nifti_real(const char* filename, const float* image, uint64_t nx, uint64_t ny, uint64_t nz,
                              uint64_t nslab, uint64_t ntr) {
  if (!filename || !image) return set_error(PG_INVALID_ARG, "NIfTI: null argument");
  uint64_t n = 0;
  PG_TRY(nifti_dims(nx, ny, nz, nslab, ntr, &n));
  return nifti_write(std::string(filename) + ".nii", image, n, nx, ny, nz, nslab, ntr);
}

pg_status pg_write_nifti_mag_phs(const char* filename, const float* image, uint64_t nx, uint64_t ny, uint64_t nz,
                                 uint64_t nslab, uint64_t ntr) {
  if (!filename || !image) return set_error(PG_INVALID_ARG, "NIfTI: null argument");
  uint64_t n = 0;
  PG_TRY(nifti_dims(nx, ny, nz, nslab, ntr, &n));
  const std::complex<float>* z = reinterpret_cast<const std::complex<float>*>(image);
  std::vector<float> mag(n), phs(n);
  for (uint64_t i = 0; i < n; ++i) {   // Armadillo abs / arg of a complex<float> column
    mag[i] = std::abs(z[i]);
    phs[i] = std::arg(z[i]);
  }
  const std::string base(filename);
  PG_TRY(nifti_write(base + "_mag.nii", mag.data(), n, nx, ny, nz, nslab, ntr));
  return nifti_write(base + "_phs.nii", phs.data(), n, nx, ny, nz, nslab, ntr);
}

}  // extern "C"
