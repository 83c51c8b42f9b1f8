#pragma once
#include "vecmem/containers/data/vector_view.hpp"
