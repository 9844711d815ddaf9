// Test-infrastructure stand-in: the reference includes this Boost.Math header
// but calls nothing from it.
#pragma once
