// Temporal drivers of the engine (radius > 0).
#include "engine.hpp"

namespace nssb {

void Engine::temporal_frame(int, const nssb_frame*, const nssb_frame*, int, int, int, nssb_frame_out*) {
    throw std::invalid_argument("nss_cuda.BM3D: radius > 0 is not available yet");
}

}  // namespace nssb
