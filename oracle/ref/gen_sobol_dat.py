"""Writes the SobolMatrix.dat the reference sampler includes (ScrambledSobolSampler/Kernel.cpp:20),
renaming the generated tables to the identifiers the reference uses (Kernel.cpp:27, 41, 47)."""
import sys

src, dst = sys.argv[1], sys.argv[2]
text = open(src).read()
text = text.replace("#pragma once", "")
text = text.replace("PB2_SOBOL_STORAGE uint32_t pb2_sobol_matrices32", "static const uint32_t sobolMatrices32")
text = text.replace("PB2_SOBOL_STORAGE uint64_t pb2_vdc_sobol_matrices_inv", "static const uint64_t vdcSobolMatricesInv")
text = text.replace("PB2_SOBOL_STORAGE uint64_t pb2_vdc_sobol_matrices", "static const uint64_t vdcSobolMatrices")
with open(dst, "w") as f:
    f.write(text)
