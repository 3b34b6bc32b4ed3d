// contract_tc.cu -- tcgen05 split-precision contraction (placeholder until the
// tensor-core kernel lands).
#include "matrix_plan.cuh"

namespace mqct {
int MatrixPlan::tc_init() {
  set_error("BF16x3 tensor-core contraction not available in this build");
  return MQCT_E_ARG;
}
int MatrixPlan::tc_execute() { return MQCT_E_ARG; }
int MatrixPlan::error_report(const double*, mqct_err_report_t*) { return MQCT_OK; }
}  // namespace mqct
