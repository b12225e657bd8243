// Instantiations of the FP32 wavefront for gcp mode (eps and beta per read):
// scalar tiles covering every read length, one per length class of the gcp
// tile table (engine.cu).
#include "fp32_kernels.cuh"

namespace phmm {

void register_fp32_gcp(std::vector<ConfigInfo>& out) {
    out.push_back(make_fp32_config<4, 16, false, false, true>());
    out.push_back(make_fp32_config<8, 16, false, false, true>());
    out.push_back(make_fp32_config<8, 20, false, false, true>());
    out.push_back(make_fp32_config<16, 16, false, false, true>());
    out.push_back(make_fp32_config<32, 16, false, false, true>());
    out.push_back(make_fp32_config<32, 32, false, false, true>());
    out.push_back(make_fp32_config<32, 32, true, false, true>());
}

}  // namespace phmm
