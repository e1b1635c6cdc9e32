// Stand-in for Falcor's Utils/Math/Common.h used by the reference unit tests
// compiled in the known-answer harness (test infrastructure only).
#pragma once
#include <cmath>
