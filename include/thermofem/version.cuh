// version.cuh -- the library version as numbers (drop-in for
// include/thermofem/version.cuh of Mgepahmge/ThermoFEM; the text form is
// tf_version()).
#pragma once

namespace thermofem {

struct Version {
    int major_{};
    int minor_{};
    int patch_{};
};

[[nodiscard]] inline Version version() noexcept { return {0, 1, 0}; }

}  // namespace thermofem
