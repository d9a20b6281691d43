// Stand-in for fmt/bundled/ostream.h (see ../fmt.h).
#pragma once
#include "../fmt.h"
