// Instantiations of the FP32 wavefront with R % 4 == 2 (tiles whose G*R falls
// on a length bound no R % 4 == 0 tile reaches with that G, e.g. 8 x 18 = 144).
#include "fp32_kernels.cuh"

namespace phmm {

void register_fp32_geven(std::vector<ConfigInfo>& out) {
    out.push_back(make_fp32_config<8, 14, false>());
    out.push_back(make_fp32_config<8, 18, false>());
    out.push_back(make_fp32_config<8, 22, false>());
    out.push_back(make_fp32_config<16, 10, false>());
    out.push_back(make_fp32_config<16, 14, false>());
    out.push_back(make_fp32_config<16, 18, false>());
}

}  // namespace phmm
