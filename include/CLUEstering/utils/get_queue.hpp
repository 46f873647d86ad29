// get_queue.hpp -- the reference's header name for clue::get_queue (defined in detail/Runtime.hpp).
#pragma once
#include "CLUEstering/detail/Runtime.hpp"
