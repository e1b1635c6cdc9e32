// Stand-in (see tests/falcor_stub/Falcor.h).
#pragma once
#include "../../Falcor.h"
