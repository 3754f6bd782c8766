// The opaque handles of the C ABI's host layer (include/blest.h): a CSC
// and a BVSS owned by the library.
#pragma once

#include "bvss.hpp"
#include "csc.hpp"

struct blest_csc {
    blest::Csc g;
};
struct blest_bvss {
    blest::Bvss b;
};
