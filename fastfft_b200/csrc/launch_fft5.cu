// Radix-5 instantiation of the length-RP launchers (lengths 5 * 2^k; see launch_fftr.cuh).
#include "launch_fftr.cuh"

namespace ffb {

FFB_DECLARE_RADIX_LAUNCHERS(, 5)

}  // namespace ffb
