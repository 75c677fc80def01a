// factory.cpp -- engine names (reference make_engine / list_engines,
// include/rtm_factory.hpp:19-23).  The reference's CPU engines are not part of
// this library; an unknown name throws like the reference's factory.
#include <stdexcept>

#include "rtm_b200_engine.hpp"

namespace rtm_b200 {

std::vector<std::string> list_engines() { return {"b200", "b200-batch", "b200-serve"}; }

std::unique_ptr<RTMEngine> make_engine(const std::string& engine_name, int requested_gpus, const B200Options* options) {
    if (requested_gpus != 1) throw std::runtime_error("the b200 engines run on one GPU (--gpus 1)");
    B200Options o = options ? *options : B200Options{};
    if (engine_name == "b200") o.mode = RTM_B200_MODE_PLAIN;
    else if (engine_name == "b200-batch") o.mode = RTM_B200_MODE_BATCH;
    else if (engine_name == "b200-serve") o.mode = RTM_B200_MODE_SERVE;
    else throw std::runtime_error("unknown or unavailable engine: '" + engine_name + "' (see --list-engines)");
    return std::make_unique<B200RTM>(o);
}

}  // namespace rtm_b200
