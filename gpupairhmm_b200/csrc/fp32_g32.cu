// Instantiations of the FP32 wavefront for groups of 32 lanes.
#include "fp32_kernels.cuh"

namespace phmm {

void register_fp32_g32(std::vector<ConfigInfo>& out) {
    out.push_back(make_fp32_config<32, 8, false>());
    out.push_back(make_fp32_config<32, 12, false>());
    out.push_back(make_fp32_config<32, 16, false>());
    out.push_back(make_fp32_config<32, 20, false>());
    out.push_back(make_fp32_config<32, 24, false>());
    out.push_back(make_fp32_config<32, 28, false>());
    out.push_back(make_fp32_config<32, 32, false>());
    out.push_back(make_fp32_config<32, 16, true>());
    out.push_back(make_fp32_config<32, 20, true>());
    out.push_back(make_fp32_config<32, 24, true>());
    out.push_back(make_fp32_config<32, 28, true>());
    out.push_back(make_fp32_config<32, 32, true>());
    out.push_back(make_fp32_config<32, 8, false, true>());
    out.push_back(make_fp32_config<32, 12, false, true>());
    out.push_back(make_fp32_config<32, 16, false, true>());
}

}  // namespace phmm
