// Instantiations of the FP32 wavefront for groups of 8 lanes.
#include "fp32_kernels.cuh"

namespace phmm {

void register_fp32_g8(std::vector<ConfigInfo>& out) {
    out.push_back(make_fp32_config<8, 8, false>());
    out.push_back(make_fp32_config<8, 12, false>());
    out.push_back(make_fp32_config<8, 16, false>());
    out.push_back(make_fp32_config<8, 20, false>());
    out.push_back(make_fp32_config<8, 24, false>());
    out.push_back(make_fp32_config<8, 28, false>());
    out.push_back(make_fp32_config<8, 32, false>());
    out.push_back(make_fp32_config<8, 8, false, true>());
    out.push_back(make_fp32_config<8, 12, false, true>());
    out.push_back(make_fp32_config<8, 16, false, true>());
}

}  // namespace phmm
