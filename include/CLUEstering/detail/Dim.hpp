// Dim.hpp -- the reference's header name for clue::Dim (defined in detail/Runtime.hpp).
#pragma once
#include "CLUEstering/detail/Runtime.hpp"
