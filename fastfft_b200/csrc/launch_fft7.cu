// Radix-7 instantiation of the length-RP launchers (lengths 7 * 2^k; see launch_fftr.cuh).
#include "launch_fftr.cuh"

namespace ffb {

FFB_DECLARE_RADIX_LAUNCHERS(, 7)

}  // namespace ffb
