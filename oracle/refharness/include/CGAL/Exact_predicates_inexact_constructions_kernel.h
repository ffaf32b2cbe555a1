// Test-harness stand-in for the CGAL header of the same name: every name the
// reference uses is provided by ../../cgal_facade.h (see there).
#pragma once
#include "../../cgal_facade.h"
