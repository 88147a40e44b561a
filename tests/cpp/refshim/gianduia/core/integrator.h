// Test shim: the reference's <gianduia/core/integrator.h> names (namespace gnd) mapped
// onto the library's mirror of the reference's plugin interface (hscene.h), so that the
// reference-side plugin source of INTEGRATION.md compiles unchanged against the mirror.
#pragma once
#include "hscene.h"

namespace gnd {
using PropertyList = gndh::PropertyList;
using Integrator = gndh::Integrator;
using Scene = gndh::Scene;
using Film = gndh::Film;
using Color3f = gnd::V3;
}  // namespace gnd
