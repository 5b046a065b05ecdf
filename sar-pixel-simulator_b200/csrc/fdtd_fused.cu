// fdtd_fused.cu -- placeholder until the fused z-marching step lands.
#include "fdtd_launch.h"

namespace fdtd {

template <class T>
bool launch_fused_step(const State<T>&, const int*, int, int, int, cudaStream_t) {
  return false;
}

template bool launch_fused_step<float>(const State<float>&, const int*, int, int, int, cudaStream_t);
template bool launch_fused_step<double>(const State<double>&, const int*, int, int, int, cudaStream_t);

}  // namespace fdtd
