// Stand-in for Cubism/StencilInfo.h: the whole stand-in lives in cubism_standin.hpp.
#pragma once
#include "../cubism_standin.hpp"
