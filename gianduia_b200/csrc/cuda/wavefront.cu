// Wavefront path-tracing engine.
#include "wavefront.h"

namespace gnd {

Wavefront::Wavefront(Context* c) : ctx_(c) {}
Wavefront::~Wavefront() = default;

}  // namespace gnd
