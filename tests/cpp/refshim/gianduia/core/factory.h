// Test shim: <gianduia/core/factory.h> (GND_REGISTER_CLASS) from the library's mirror.
#pragma once
#include "hscene.h"
