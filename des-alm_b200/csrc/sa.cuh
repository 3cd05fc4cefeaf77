// sa.cuh -- Spalart-Allmaras sub-iterations on the fine level (des_eddy).
#pragma once
#include "common.cuh"

namespace desalm {

// fine-level FP64 work arrays of the SA model
struct SaWork {
  static const int NARR = 12;
  double* a[NARR];
};

}  // namespace desalm
