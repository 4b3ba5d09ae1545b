// config_c.h — FluidConfig (include/core/config.h) <-> pbf_fluid_config
// (include/pbf_b200.h), field by field.
#ifndef PBF_B200_HOST_CONFIG_C_H
#define PBF_B200_HOST_CONFIG_C_H

#include "../../include/core/config.h"
#include "../../include/pbf_b200.h"

namespace pbfhost {
void fluid_config_to_c(const FluidConfig& p, pbf_fluid_config* out);
FluidConfig fluid_config_from_c(const pbf_fluid_config& c);
}  // namespace pbfhost

#endif
