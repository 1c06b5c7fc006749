// Specialised explicit line operators on double fields.
#define CHS_STENCIL_T double
#include "chs_stencil_impl.cuh"
