// design_inst_loss.cu -- row passes of the surrogate's phase loss and gradient,
// every length and shape variant.
#define DOE_DESIGN_INSTANTIATE
#include "design_ops.cuh"

namespace doe {
DOE_DESIGN_ROW_INST(RowLossField)
DOE_DESIGN_ROW_INST(RowPhaseGrad)
}  // namespace doe
