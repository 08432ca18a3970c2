// The service's molecule description (include/lio_serve.h) as a lio::System.
#pragma once
#include "../../include/lio_serve.h"
#include "system.h"

namespace lio {
// checks the description and copies it into a System (atoms, basis, functional)
System system_from_molecule(const lio_molecule* d);
}  // namespace lio
