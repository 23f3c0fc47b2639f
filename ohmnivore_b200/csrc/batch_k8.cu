// Batch kernel instantiations for 8 lane(s) per row.
#include "batch_kernel.cuh"

namespace ohm {

BatchFn batch_kernel_lpr8(int shape) {
    switch (shape) {
        case 0: return batch_solver<8, kBatchShapes[0].block, kBatchShapes[0].min_blocks>;
        case 1: return batch_solver<8, kBatchShapes[1].block, kBatchShapes[1].min_blocks>;
        default: return batch_solver<8, kBatchShapes[2].block, kBatchShapes[2].min_blocks>;
    }
}

}  // namespace ohm
