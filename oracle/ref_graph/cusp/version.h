// ORACLE — test infrastructure only: see shim.h.  The shim provides the
// post-0.5 CUSP interface (cusp::offsets_to_indices, cusp::blas::fill).
#pragma once
#define CUSP_VERSION 500
