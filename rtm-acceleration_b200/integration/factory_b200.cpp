// factory_b200.cpp -- the reference's engine registry (its make_engine /
// list_engines interface, include/rtm_factory.hpp:19-23) with the B200 engines
// registered beside its CPU engines, the way src/rtm/factory.cpp:17-54 of the
// reference registers each engine: one name, one constructor.  Replaces that
// file in the ref-b200 build of oracle/Makefile; every other reference source
// is compiled unmodified.
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cpu_opt.hpp"
#include "rtm_cpu.hpp"
#include "rtm_factory.hpp"

namespace rtm {

std::unique_ptr<RTMEngine> make_b200_engine(const std::string& name);   // b200_engine.cpp

std::unique_ptr<RTMEngine> make_engine(const std::string& engine_name, int requested_gpus) {
    (void)requested_gpus;
    if (engine_name == "cpu") return std::make_unique<CPUReferenceRTM>();
    if (engine_name == "cpu-opt") return std::make_unique<CPUOptimizedRTM>();
    if (auto e = make_b200_engine(engine_name)) return e;
    throw std::runtime_error("unknown or unavailable engine: '" + engine_name + "' (see --list-engines)");
}

std::vector<std::string> list_engines() { return {"cpu", "cpu-opt", "b200", "b200-batch", "b200-serve"}; }

}  // namespace rtm
