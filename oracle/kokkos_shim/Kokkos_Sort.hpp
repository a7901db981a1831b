// Kokkos_Sort.hpp -- TEST INFRASTRUCTURE ONLY.
// Included by the Jet reference sources but not used by them; the Kokkos
// stand-in in this directory provides nothing more for it.
#pragma once
#include "Kokkos_Core.hpp"
