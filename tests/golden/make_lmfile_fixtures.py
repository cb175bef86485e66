"""Copies the reference's HDF5 test fixtures (testing/data/lm/io/hdf5/*.h5,
written by libhdf5 and Matlab; 5 B to 10 KB each) into tests/golden/lmfile/,
byte for byte, so that the `.lm` reader is checked against files a real HDF5
library wrote.  Run from the repository root with the reference checkout as
the argument."""
import os
import shutil
import sys

NAMES = ["SimulationFile_1.h5", "SimulationFile_2.h5", "SimulationFile_3.h5", "SimulationFile_GetDiffusionModel.h5",
         "SimulationFile_GetReactionModel.h5", "SimulationFile_GetReactionModel_NoReactionCount.h5",
         "SimulationFile_GetReactionModel_Noise.h5", "SimulationFile_GetSpatialModelObjects.h5"]

if __name__ == "__main__":
    src = os.path.join(sys.argv[1], "testing", "data", "lm", "io", "hdf5")
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lmfile")
    os.makedirs(dst, exist_ok=True)
    for n in NAMES:
        shutil.copyfile(os.path.join(src, n), os.path.join(dst, n))
