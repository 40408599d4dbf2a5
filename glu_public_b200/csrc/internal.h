// Internal declarations shared by the host and device sources of libglu_b200.
#pragma once

#include <cstdint>
#include <cstdio>
#include <vector>

#include "glu_b200.h"

namespace glu {

// Records a thread-local message for glu_last_error() and returns `code`.
int set_error(int code, const char* fmt, ...);

int symbolic_fill(uint32_t n, const uint32_t* ap, const uint32_t* ai, std::vector<uint32_t>& cp,
                  std::vector<uint32_t>& ri, std::vector<uint32_t>& lp);
void symbolic_csr(uint32_t n, const std::vector<uint32_t>& cp, const std::vector<uint32_t>& ri,
                  std::vector<uint32_t>& rp, std::vector<uint32_t>& ci, std::vector<uint32_t>& dp);
int32_t symbolic_levels(uint32_t n, const std::vector<uint32_t>& cp,
                        const std::vector<uint32_t>& ri, const std::vector<uint32_t>& lp,
                        const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci,
                        const std::vector<uint32_t>& dp, std::vector<int32_t>& lev_ptr,
                        std::vector<int32_t>& lev_idx);

}  // namespace glu
