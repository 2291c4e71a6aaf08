// design_inst_col_asm.cu -- image-plane propagation column passes of the design
// loops (forward and back), every length and shape variant.
#define DOE_DESIGN_INSTANTIATE
#include "design_ops.cuh"

namespace doe {
DOE_DESIGN_COL_INST(ColAsmTab<false>)
DOE_DESIGN_COL_INST(ColAsmTab<true>)
}  // namespace doe
