// Test shim: <gianduia/core/fileResolver.h> from the library's mirror.
#pragma once
#include "hscene.h"

namespace gnd {
using FileResolver = gndh::FileResolver;
}  // namespace gnd
