// Name-keyed registry of matrix-profile algorithm variants.
#include "matprof_algo.hpp"

#include <sstream>

namespace matrix_profile {

MatProfImplFactory& MatProfImplFactory::getInstance() {
    static MatProfImplFactory instance;  // built on first use, thread-safe
    return instance;
}

bool MatProfImplFactory::register_impl(const std::string& name, Creator creator_fn) {
    return registrations_.emplace(name, creator_fn).second;
}

std::string MatProfImplFactory::get_available_implementations() const {
    std::ostringstream os;
    for (const auto& kv : registrations_) os << kv.first << " ";
    return os.str();
}

std::unique_ptr<IMatProfAlgo> MatProfImplFactory::create(const std::string& algo_name) const {
    return registrations_.at(algo_name)();
}

}  // namespace matrix_profile
