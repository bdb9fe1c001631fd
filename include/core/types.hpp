// Forwarding header at the reference's include path (src/core/types.hpp).
#pragma once
#include "../swiftimpute/imputer.hpp"
