// Forwarding header at the reference's include path (src/api/imputer.hpp), so
// callers written against the reference compile unchanged with -I include.
#pragma once
#include "../swiftimpute/imputer.hpp"
