// Oracle test infrastructure: host stand-in for <optix.h> (see optix_types.h).
#pragma once
#include "optix_types.h"
