// core/Config.h — the spelling used by the reference sources (#include "core/Config.h").
#include "core/config.h"
