// Built in place of anukulan's src/anukulan/cuda_backend.cu, this file makes
// anukulan::cuda_backend() (src/anukulan/backend.hpp:233-236) return the
// LinAlgBackend adapter over this library's kernels (include/
// anu_b200_backend.hpp). With ANUKULAN_WITH_CUDA defined, anukulan's
// default_backend() (backend.cpp:209-221) then hands that adapter to every
// solve_pdhg that names no backend, and falls back to the CPU when no device
// is present, exactly as with the reference's own CUDA backend.
//
// Link: anukulan's objects + this file + -lanu_pdhg (no nvcc step, no
// device code of anukulan's own).

#include "anu_b200_backend.hpp"

namespace anukulan {

const LinAlgBackend& cuda_backend() { return anu_b200::backend(); }

}  // namespace anukulan
