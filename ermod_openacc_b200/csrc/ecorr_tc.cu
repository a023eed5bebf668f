// ecorr_tc.cu -- placeholder until the tcgen05 INT8 path lands.
#include "engine.cuh"
namespace erm {
int ecorr_tc_available() { return 0; }
size_t ecorr_tc_workspace(int, int) { return 0; }
int launch_ecorr_tc(const DeviceState&, int, int, int, int, int, int, void*, size_t, cudaStream_t) { return -1; }
}  // namespace erm
