"""Generate tests/golden/nifti_magphs.npz: NIfTI files written through the
reference's own header definition.

A small C++ program (written below) includes PowerGrid's Support/nifti1.h from
the reference tree, fills `nifti_1_header` field by field as
writeNiftiRealImage does (processNIFTI.hpp:44-86; the struct is zeroed first,
since the reference leaves the other fields uninitialised), takes abs/arg of a
complex image as writeNiftiMagPhsImage does (processNIFTI.hpp:106-107) and
writes header, 4-byte extender and float32 voxels (:88-99).  The resulting
bytes pin the library's writer, which lays the header out by byte offset.

Run where the reference tree exists, with PG_REFERENCE_ROOT naming the
reference project's root (the directory holding Support/ and PowerGrid/):
    PG_REFERENCE_ROOT=<root> python tests/golden/make_nifti_golden.py
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _ref_support() -> str:
    root = os.environ.get("PG_REFERENCE_ROOT")
    if not root:
        raise SystemExit("set PG_REFERENCE_ROOT to the reference project's root (holding Support/nifti1.h)")
    return os.path.join(root, "Support")

PROGRAM = r'''
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>
#include "nifti1.h"

static void write_real(const std::string& fn, const std::vector<float>& v, int nx, int ny, int nz, int nslab,
                       int ntr) {
  nifti_1_header hdr;
  std::memset(&hdr, 0, sizeof(hdr));
  nifti1_extender pad = {{0, 0, 0, 0}};
  hdr.sizeof_hdr = 348;
  hdr.dim[0] = 3;
  hdr.dim[1] = nx; hdr.dim[2] = ny; hdr.dim[3] = nz; hdr.dim[4] = nslab; hdr.dim[5] = ntr;
  hdr.dim[6] = 1; hdr.dim[7] = 1;
  hdr.datatype = NIFTI_TYPE_FLOAT32;
  hdr.bitpix = 32;
  hdr.pixdim[0] = 1.0; hdr.pixdim[1] = 1.0; hdr.pixdim[2] = 1.0; hdr.pixdim[3] = 1.0;
  hdr.vox_offset = 352.0f;
  hdr.scl_slope = 100.0;
  hdr.xyzt_units = NIFTI_UNITS_MM;
  std::strncpy(hdr.magic, "n+1\0", 4);
  std::ofstream o(fn + ".nii", std::ios::binary);
  o.write((const char*)&hdr, 348);
  o.write((const char*)&pad, 4);
  o.write((const char*)v.data(), v.size() * sizeof(float));
}

int main(int argc, char** argv) {
  const int nx = atoi(argv[2]), ny = atoi(argv[3]), nz = atoi(argv[4]), nslab = atoi(argv[5]), ntr = atoi(argv[6]);
  const size_t n = (size_t)nx * ny * nz * nslab * ntr;
  std::vector<std::complex<float>> z(n);
  std::FILE* f = std::fopen(argv[1], "rb");
  if (std::fread(z.data(), sizeof(z[0]), n, f) != n) return 1;
  std::fclose(f);
  std::vector<float> mag(n), phs(n);
  for (size_t i = 0; i < n; ++i) { mag[i] = std::abs(z[i]); phs[i] = std::arg(z[i]); }
  write_real(std::string(argv[7]) + "_mag", mag, nx, ny, nz, nslab, ntr);
  write_real(std::string(argv[7]) + "_phs", phs, nx, ny, nz, nslab, ntr);
  return 0;
}
'''


def main():
    nx, ny, nz, nslab, ntr = 6, 6, 2, 1, 2
    n = nx * ny * nz * nslab * ntr
    rng = np.random.default_rng(31)
    z = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    # arg's branch points and zero: 0, negative reals with +0 and -0 imaginary parts
    z[0] = 0
    z[1] = complex(-2.0, 0.0)
    z[2] = np.complex64(complex(-3.0, -0.0))
    z[3] = complex(0.0, -1.5)
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "nifti_ref.cpp")
        with open(src, "w") as f:
            f.write(PROGRAM)
        exe = os.path.join(d, "nifti_ref")
        subprocess.run(["g++", "-std=c++17", "-O0", "-I" + _ref_support(), src, "-o", exe], check=True)
        zin = os.path.join(d, "z.bin")
        z.tofile(zin)
        base = os.path.join(d, "img")
        subprocess.run([exe, zin, str(nx), str(ny), str(nz), str(nslab), str(ntr), base], check=True)
        mag = np.fromfile(base + "_mag.nii", np.uint8)
        phs = np.fromfile(base + "_phs.nii", np.uint8)
    np.savez_compressed(os.path.join(HERE, "nifti_magphs.npz"), z=z, dims=np.array([nx, ny, nz, nslab, ntr]),
                        mag_file=mag, phs_file=phs)
    print(f"nifti_magphs.npz: {mag.size} + {phs.size} bytes")


if __name__ == "__main__":
    main()
