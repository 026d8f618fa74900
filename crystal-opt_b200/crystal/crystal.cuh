// crystal.cuh -- block-wide device functions for star-join drivers, rebuilt for
// sm_100a with the same names, signatures and semantics as the reference's
// crystal/crystal.cuh umbrella (crystal/crystal.cuh:25-32), so query drivers
// written against it compile unchanged (put this directory first on the include
// path).
#pragma once

#include "load.cuh"
#include "pred.cuh"
#include "store.cuh"
#include "reduce.cuh"
#include "join.cuh"
#include "term.cuh"
#include "bloom.cuh"
