/* TEST INFRASTRUCTURE ONLY: VTK stand-in, see m3d_vtk_stub.h */
#include "m3d_vtk_stub.h"
