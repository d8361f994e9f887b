// Wavefront path tracer (declarations shared by the render translation units).
#pragma once
#include "fl_internal.h"
