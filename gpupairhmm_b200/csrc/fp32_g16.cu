// Instantiations of the FP32 wavefront for groups of 16 lanes.
#include "fp32_kernels.cuh"

namespace phmm {

void register_fp32_g16(std::vector<ConfigInfo>& out) {
    out.push_back(make_fp32_config<16, 8, false>());
    out.push_back(make_fp32_config<16, 12, false>());
    out.push_back(make_fp32_config<16, 16, false>());
    out.push_back(make_fp32_config<16, 20, false>());
    out.push_back(make_fp32_config<16, 24, false>());
    out.push_back(make_fp32_config<16, 28, false>());
    out.push_back(make_fp32_config<16, 32, false>());
    out.push_back(make_fp32_config<16, 32, true>());
    out.push_back(make_fp32_config<16, 8, false, true>());
    out.push_back(make_fp32_config<16, 10, false, true>());
    out.push_back(make_fp32_config<16, 12, false, true>());
    out.push_back(make_fp32_config<16, 16, false, true>());
}

}  // namespace phmm
