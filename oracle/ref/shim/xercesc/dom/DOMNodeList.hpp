#include "dom_shim.hpp"
