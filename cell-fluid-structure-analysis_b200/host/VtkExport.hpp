// io::exportToVtk for the fluid solver (include/IO/VtkExport.hpp:20-21, src/IO/VtkExport.cpp:238-268):
// the same legacy-VTK text, written from the device fields by cfsa_ns_write_vtk (asynchronous
// device-to-host copies overlapped with formatting the mesh part). `fields` (new) appends
// per-vertex boundary-force vectors: CFSA_VTK_SHEAR_STRESS, CFSA_VTK_PRESSURE_FORCES.
#pragma once

#include "NavierStokes.hpp"

#include <iostream>
#include <string>

namespace io {
inline void exportToVtk(const std::string &filename, const NavierStokesSolver &ns_solver,
                        double scale = 1.0, int fields = 0) {
  if (!ns_solver.handle()) return;
  const int code = cfsa_ns_write_vtk(ns_solver.handle(), filename.c_str(), scale, fields);
  if (code != CFSA_OK)
    std::cerr << "[IO] Failed to write " << filename << ": " << cfsa_ns_last_error(ns_solver.handle())
              << std::endl;
}
}  // namespace io
