// Minimal stand-in for Falcor's Core/Macros.h, so that reference sources that
// only need the export macro compile on their own (test infrastructure).
#pragma once
#define FALCOR_API
