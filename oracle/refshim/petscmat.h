/* oracle build of the reference sources: PETSc/SLEPc names come from refshim.h */
#include "refshim.h"
