// sbx_oracle_f64.cpp — CPU ORACLE (test infrastructure) in double precision: the oracle's
// restatement of the System methods and harness steps compiled with every `float` (store
// arrays, forces, drag, orientations, accumulators, the float casts of the reference's
// arithmetic) evaluated as `double`, and the portable transcendentals of sbx_math.h. The
// FP32 kernels equal the FP32 oracle bit for bit, so comparing the FP32 oracle with this
// build states the error of the FP32 kernels against an FP64 evaluation of the same
// algorithm. The scene structs of include/softbox_b200.h then hold double pointers.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define float double
#define SBX_ORACLE_DEVMATH 1
#include "sbx_oracle.cpp"
#include "sbx_oracle_dense.cpp"
