// sqlfloat.cuh — SQL float8 arithmetic on the device: map/arithmetic.rs:
// 49-79 (float8_pl / _mi / _mul / _div): a finite result that overflows,
// a non-zero result that underflows to zero, and division by zero are
// errors, not silent infinities or zeros.
#pragma once

#include "../../include/warren_cuda.h"

namespace wc {

enum FloatOp { F_ADD = 0, F_SUB = 1, F_MUL = 2, F_DIV = 3 };

template <int OP> __host__ __device__ inline int32_t sql_float(double a, double b, double* o) {
  if (OP == F_DIV && b == 0.0 && !(a != a)) return WC_DIVISION_BY_ZERO;
  double r;
  if (OP == F_ADD) r = a + b;
  else if (OP == F_SUB) r = a - b;
  else if (OP == F_MUL) r = a * b;
  else r = a / b;
  bool finite_operands = OP == F_DIV ? !isinf(a) : (!isinf(a) && !isinf(b));
  if (isinf(r) && finite_operands) return WC_FLOAT_OVERFLOW;
  bool underflowed = OP == F_MUL ? (a != 0.0 && b != 0.0)
                                 : (OP == F_DIV ? (a != 0.0 && !isinf(b)) : false);
  if (r == 0.0 && underflowed) return WC_FLOAT_UNDERFLOW;
  *o = r;
  return 0;
}

}  // namespace wc
