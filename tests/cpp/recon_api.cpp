// Drives the C++ operator API (include/powergrid/PowerGrid.hpp) the way the
// reference's PowerGridIsmrmrd driver does (PowerGridIsmrmrd.cpp:244-264):
// Gnufft -> TimeSegmentation -> SENSE -> operator*, operator/, reconSolve,
// then the direct-reconstruction helpers, the spatial interpolation and a
// low-rank model over the same operator, and the same image through the
// request server.
// Inputs and outputs are raw little-endian files in the directory argv[1]
// (written and checked by tests/test_cpp_api.py).
#include <complex>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "powergrid/PowerGrid.hpp"

using cx = std::complex<float>;

template <typename T>
pg::Col<T> load(const std::string& path, pg::uword n) {
  pg::Col<T> c(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(c.memptr()), n * sizeof(T));
  if (!f) throw std::runtime_error("cannot read " + path);
  return c;
}

template <typename T>
void save(const std::string& path, const pg::Col<T>& c) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(c.memptr()), c.size() * sizeof(T));
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string d = argv[1];
  std::ifstream meta(d + "/meta.txt");
  pg::uword nx, ny, nz, M, L, nc, niter;
  float beta;
  meta >> nx >> ny >> nz >> M >> L >> nc >> niter >> beta;
  const pg::uword N = nx * ny * nz;
  try {
    auto kx = load<float>(d + "/kx.bin", M), ky = load<float>(d + "/ky.bin", M), kz = load<float>(d + "/kz.bin", M);
    auto t = load<float>(d + "/t.bin", M);
    auto fm = load<float>(d + "/fm.bin", N);
    auto sm = load<cx>(d + "/smap.bin", N * nc);
    auto x = load<cx>(d + "/x.bin", N);
    auto data = load<cx>(d + "/data.bin", M * nc);
    pg::Col<float> ix(N), iy(N), iz(N);
    pg::Gnufft<float> G(M, 2.0f, nx, ny, nz, kx, ky, kz, ix, iy, iz);
    pg::TimeSegmentation<float, pg::Gnufft<float>> A(G, fm, t, M, N, L, 1, 1);
    pg::SENSE<float, pg::TimeSegmentation<float, pg::Gnufft<float>>> S(A, sm, M, N, nc);
    pg::QuadPenalty<float> R(nx, ny, nz, beta);
    pg::Col<cx> y = S * x;
    pg::Col<cx> xa = S / data;
    pg::Col<cx> img = pg::reconSolve<float>(data, S, R, kx, ky, kz, nx, ny, nz, t, niter);
    save(d + "/y_out.bin", y);
    save(d + "/xadj_out.bin", xa);
    save(d + "/img_out.bin", img);
    // direct reconstruction (reconSupport/directRecon.cpp): density
    // compensation, per-coil gridded images, coil combination
    pg::Col<float> dcf = pg::calc3DDensityCompensation<float>(kx, ky, kz, nx, nz);
    pg::Col<cx> coil = pg::gridCoilImages<float>(G, dcf, data, nc);
    pg::Col<float> sos = pg::calcSumOfSquaresImage<float, pg::Col<float>>(coil, nc);
    save(d + "/dcf_out.bin", dcf);
    save(d + "/sos_out.bin", sos);
    // spatial interpolation round trip on the oversampled grid
    pg::Col<cx> y0(M);  // the first coil's samples
    for (pg::uword i = 0; i < M; ++i) y0.memptr()[i] = y.memptr()[i];
    pg::Col<cx> grid = G.adjointSpatialInterp(y0);
    save(d + "/interp_out.bin", G.forwardSpatialInterp(grid));
    // the low-rank model as lowRank/oscillateRecon.cpp:256-265 composes it:
    // two repetitions through the same SENSE operator, identity basis
    {
      using Sop = pg::SENSE<float, pg::TimeSegmentation<float, pg::Gnufft<float>>>;
      Sop* All[2] = {&S, &S};
      pg::Col<cx> v(4, cx(0, 0));
      v[0] = cx(1, 0);
      v[3] = cx(1, 0);
      pg::LRobj<float, Sop> Alr(N, M * nc, 2, 2, v, All);
      pg::Col<cx> x2(2 * N), d2(2 * M * nc), x0(2 * N, cx(0, 0));
      for (pg::uword i = 0; i < N; ++i) x2[i] = x2[N + i] = x[i];
      for (pg::uword i = 0; i < M * nc; ++i) d2[i] = d2[M * nc + i] = data[i];
      save(d + "/ylr_out.bin", Alr * x2);
      pg::R_lowRank<float, pg::QuadPenalty<float>> Rlr(R, 2, 2, v);
      pg::Col<float> W(2 * M * nc, 1.0f);
      pg::Col<cx> xlr = pg::solve_pwls_pcg<float, pg::LRobj<float, Sop>, pg::R_lowRank<float, pg::QuadPenalty<float>>>(
          x0, Alr, W, d2, Rlr, 3);
      save(d + "/xlr_out.bin", xlr);
    }
    // the reconstructed image as NIfTI magnitude and phase (processNIFTI.hpp:103-117)
    pg::writeNiftiMagPhsImage<float>(d + "/img", img, nx, ny, nz);
    // an acquisition list of two shots, gathered back into one image's data
    {
      const pg::uword half = M / 2;
      std::vector<float> tr(4 * M);
      for (pg::uword s = 0; s < M; ++s) {
        tr[4 * s] = kx[s]; tr[4 * s + 1] = ky[s]; tr[4 * s + 2] = kz[s]; tr[4 * s + 3] = t[s];
      }
      std::vector<cx> a0(nc * half), a1(nc * half);
      for (pg::uword c = 0; c < nc; ++c)
        for (pg::uword s = 0; s < half; ++s) {
          a0[c * half + s] = data[c * M + s];
          a1[c * half + s] = data[c * M + half + s];
        }
      std::vector<pg_acquisition> acqs(2);
      for (int k = 0; k < 2; ++k) {
        acqs[k] = pg_acquisition{(uint32_t)k, 0, 0, 0, 0, 0, 0, (uint32_t)half, (uint32_t)nc, 4,
                                 reinterpret_cast<const float*>(k ? a1.data() : a0.data()), tr.data() + 4 * half * k};
      }
      pg::acqTracking track(acqs, pg_encoding_limits{2, 1, 1, 1, 1, 1, 1});
      pg::Col<cx> gd;
      pg::Col<float> gkx, gky, gkz, gt;
      pg::getCompleteISMRMRDAcqData<float>(track, 0, 0, 0, 0, 0, gd, gkx, gky, gkz, gt);
      save(d + "/gather_data.bin", gd);
      save(d + "/gather_kx.bin", gkx);
      // the same image served: as a request, and as the driver's loop over the index
      pg::Server srv(8ull << 30, 2);
      pg::Col<cx> sreq(N), sacq(N);
      const pg_request rq{nx, ny, nz, 1, nc, M, L, niter, beta, kx.memptr(), ky.memptr(), kz.memptr(), t.memptr(),
                          fm.memptr(), reinterpret_cast<const float*>(sm.memptr()),
                          reinterpret_cast<const float*>(data.memptr()), reinterpret_cast<float*>(sreq.memptr())};
      const pg_acq_request aq{nx, ny, nz, L, niter, beta, fm.memptr(), reinterpret_cast<const float*>(sm.memptr()),
                              reinterpret_cast<float*>(sacq.memptr())};
      const uint64_t t1 = srv.submit(rq), t2 = srv.submit(track, aq);
      for (const uint64_t tk : {t1, t2}) {
        const pg_request_stats st = srv.wait(tk);
        if (st.status != PG_OK) throw pg::Error(st.status, st.error);
      }
      save(d + "/served_req.bin", sreq);
      save(d + "/served_acq.bin", sacq);
    }
  } catch (const pg::Error& e) {
    std::fprintf(stderr, "pg error: %s\n", e.what());
    return 1;
  }
  return 0;
}
