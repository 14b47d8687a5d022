// Stand-in for Cubism/BlockLabMPI.h: the whole stand-in lives in cubism_standin.hpp.
#pragma once
#include "../cubism_standin.hpp"
