"""PowerGrid's system-operator path on B200 (sm_100a).

The compute lives in libpowergrid_b200.so (CUDA C++, C ABI in
include/powergrid_b200.h).  This package is the Python host mirror of the
reference's operator interface; importing it does not touch the GPU.
"""
from .operators import (SENSE, Gdft, GdftR2, Gnufft, LRobj, QuadPenalty, R_lowRank, TimeSegmentation, TVPenalty,
                        calc3DDensityCompensation, calcSumOfSquaresImage, gridCoilImages, init, pcg_resume,
                        pcg_state_save, pcSENSE, pcSenseTimeSeg, reconSolve, solve_pwls_pcg, solve_pwls_pcg_device)

__all__ = ["Gnufft", "Gdft", "GdftR2", "TimeSegmentation", "SENSE", "pcSenseTimeSeg", "pcSENSE", "LRobj", "QuadPenalty",
           "calc3DDensityCompensation", "gridCoilImages", "calcSumOfSquaresImage", "TVPenalty", "R_lowRank",
           "solve_pwls_pcg", "solve_pwls_pcg_device", "pcg_state_save", "pcg_resume", "reconSolve", "init"]
