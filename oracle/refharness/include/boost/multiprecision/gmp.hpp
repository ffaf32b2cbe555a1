// Test-harness stand-in: the reference includes this header but uses no name
// from it on the interpolation path.
#pragma once
