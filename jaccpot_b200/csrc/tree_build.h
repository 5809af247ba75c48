// Host-side prepare (tree + interaction lists); see tree_build.cpp.
#pragma once
#include "../../include/jaccpot_b200.h"
