// kpp_b200 CUDA target of the KPP generator: the sparse-LU template pasted
// into <root>_LinearAlgebra.cu (the C target pastes util/sutil.c there).
//
// KppDecomp (util/sutil.c:2-23): in-place no-pivot LU of one cell's matrix in
// the LU pattern, row by row through a dense work row, the multiplier of each
// eliminated entry stored in its place; returns k+1 when the diagonal entry
// of row k is zero on entry to its elimination, 0 on success.  The same
// operations in the same order as the C routine, as a device template over
// the matrix argument (a pointer or a strided view of per-cell storage); the
// LU tables are the device arrays of <root>_JacobianSP.cu.
template <class TJ>
__device__ __forceinline__ int KppDecomp(TJ&& JVS)
{
  double W[KPP_NVAR];
  for (int k = 0; k < KPP_NVAR; k++) {
    const int dk = LU_DIAG[k], first = LU_CROW[k], last = LU_CROW[k + 1];
    if (JVS[dk] == 0.0) return k + 1;
    for (int kk = first; kk < last; kk++) W[LU_ICOL[kk]] = JVS[kk];
    for (int kk = first; kk < dk; kk++) {
      const int j = LU_ICOL[kk];
      const double a = -W[j] / JVS[LU_DIAG[j]];
      W[j] = -a;
      for (int jj = LU_DIAG[j] + 1; jj < LU_CROW[j + 1]; jj++) {
        const int c = LU_ICOL[jj];
        W[c] = W[c] + a * JVS[jj];
      }
    }
    for (int kk = first; kk < last; kk++) JVS[kk] = W[LU_ICOL[kk]];
  }
  return 0;
}
