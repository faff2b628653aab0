// ORACLE — test infrastructure only: see shim.h.
#pragma once
#include <cusp/shim.h>
