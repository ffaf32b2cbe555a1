// Test-harness stand-in: the reference's kd-tree includes this header but
// uses nothing from it.
#pragma once
