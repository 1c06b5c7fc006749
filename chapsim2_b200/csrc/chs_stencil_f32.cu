// Specialised explicit line operators on float fields.
#define CHS_STENCIL_T float
#include "chs_stencil_impl.cuh"
