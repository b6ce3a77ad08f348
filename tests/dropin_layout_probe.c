/* Test helper (compiled by tests/test_dropin.py): prints the size and the
 * field offsets of the reference-ABI structs, and puts the drop-in Init /
 * Deinit functions into a KernelFunctionsType table exactly as a row of
 * LBM-Bench's GKernels[] would (src/lbm.c:33-41). Compiled once against the
 * reference's own src/lbm.h (included first, so lbm_b200_dropin.h uses the
 * reference's types) and once against lbm_b200_dropin.h alone; the two
 * outputs must be identical. */
#include <stddef.h>
#include <stdio.h>

#ifdef WITH_REFERENCE_HEADER
#include "lbm.h"
#endif
#include "lbm_b200_dropin.h"

#define OFF(T, f) printf(#T "." #f " %zu\n", offsetof(T, f))

static KernelFunctionsType table[] = {
  { "cuda-pull-soa", kernelInitCudaPullSoA, kernelDeinitCuda },
  { "cuda-push-soa", kernelInitCudaPushSoA, kernelDeinitCuda },
  { "cuda-aa-soa", kernelInitCudaAaSoA, kernelDeinitCuda },
};

int main(void)
{
  printf("sizeof PdfType %zu\n", sizeof(PdfType));
  printf("sizeof LatticeDescType %zu\n", sizeof(LatticeDescType));
  OFF(LatticeDescType, Dims);
  OFF(LatticeDescType, Lattice);
  OFF(LatticeDescType, nCells);
  OFF(LatticeDescType, nFluid);
  OFF(LatticeDescType, nObst);
  OFF(LatticeDescType, PeriodicX);
  OFF(LatticeDescType, PeriodicZ);
  OFF(LatticeDescType, Name);
  printf("sizeof CaseDataType %zu\n", sizeof(CaseDataType));
  OFF(CaseDataType, Omega);
  OFF(CaseDataType, XForce);
  OFF(CaseDataType, MaxIterations);
  OFF(CaseDataType, StatisticsModulus);
  printf("sizeof KernelDataType %zu\n", sizeof(KernelDataType));
  OFF(KernelDataType, Pdfs);
  OFF(KernelDataType, PdfsActive);
  OFF(KernelDataType, Dims);
  OFF(KernelDataType, GlobalDims);
  OFF(KernelDataType, Offsets);
  OFF(KernelDataType, BounceBackPdfsSrc);
  OFF(KernelDataType, BounceBackPdfsDst);
  OFF(KernelDataType, nBounceBackPdfs);
  OFF(KernelDataType, Blk);
  OFF(KernelDataType, Iteration);
  OFF(KernelDataType, LoopBalance);
  OFF(KernelDataType, Duration);
  OFF(KernelDataType, GetNode);
  OFF(KernelDataType, SetNode);
  OFF(KernelDataType, BoundaryConditionsGetPdf);
  OFF(KernelDataType, BoundaryConditionsSetPdf);
  OFF(KernelDataType, Kernel);
  printf("sizeof KernelFunctionsType %zu\n", sizeof(KernelFunctionsType));
  printf("rows %zu\n", sizeof(table) / sizeof(table[0]));
  return 0;
}
