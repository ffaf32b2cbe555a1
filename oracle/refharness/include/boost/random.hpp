// Test-harness stand-in.
#pragma once
#include "random/mersenne_twister.hpp"
#include "random/uniform_real.hpp"
#include "random/variate_generator.hpp"
