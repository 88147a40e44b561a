// Wavefront path-tracing engine (declared here, defined in wavefront.cu).
#pragma once
#include "runtime.h"

namespace gnd {

class Wavefront {
public:
    explicit Wavefront(Context* c);
    ~Wavefront();

private:
    Context* ctx_;
};

}  // namespace gnd
