// Instantiations of the FP32 wavefront for groups of 4 lanes.
#include "fp32_kernels.cuh"

namespace phmm {

void register_fp32_g4(std::vector<ConfigInfo>& out) {
    out.push_back(make_fp32_config<4, 4, false>());
    out.push_back(make_fp32_config<4, 8, false>());
    out.push_back(make_fp32_config<4, 12, false>());
    out.push_back(make_fp32_config<4, 16, false>());
    out.push_back(make_fp32_config<4, 20, false>());
    out.push_back(make_fp32_config<4, 24, false>());
    out.push_back(make_fp32_config<4, 28, false>());
    out.push_back(make_fp32_config<4, 32, false>());
    out.push_back(make_fp32_config<4, 8, false, true>());
    out.push_back(make_fp32_config<4, 12, false, true>());
    out.push_back(make_fp32_config<4, 16, false, true>());
}

}  // namespace phmm
