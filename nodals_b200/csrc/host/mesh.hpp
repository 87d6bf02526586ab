// Tetrahedral mesh in the form the SIMPLE setup consumes.
//
// Cell construction follows the reference reader
// (gpu/serial_cuda/foam_mesh_g2.hpp:55-57): a cell's four vertices are the
// union of its four triangular faces sorted ascending, with vertices 1 and 2
// swapped when the Jacobian determinant is negative; opp[c][i] is the face
// of cell c that does not contain local vertex i.  Face numbering drives the
// numbering of face-bubble unknowns, so every reader here produces the same
// canonical face order for the same cells (see canonical_faces in mesh.cpp).
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace nds {

struct Patch {
  std::string name;
  int start = 0;
  int count = 0;
};

struct Mesh {
  std::vector<double> xyz;                    // 3 * n_points
  std::vector<std::array<int32_t, 3>> faces;  // triangles
  std::vector<int32_t> owner, neighbour;      // neighbour.size() == internal faces
  std::vector<Patch> patches;
  std::vector<int32_t> face_patch;            // -1 for internal faces
  std::vector<std::array<int32_t, 4>> tets;   // sorted, positively oriented
  std::vector<std::array<int32_t, 4>> opp;    // face opposite local vertex i

  int n_points() const { return (int)(xyz.size() / 3); }
  int n_faces() const { return (int)faces.size(); }
  int n_internal() const { return (int)neighbour.size(); }
  int n_cells() const { return (int)tets.size(); }
  double x(int v) const { return xyz[3 * (size_t)v]; }
  double y(int v) const { return xyz[3 * (size_t)v + 1]; }
  double z(int v) const { return xyz[3 * (size_t)v + 2]; }
  int patch_index(const std::string& name) const;
};

// 3x3 determinant / inverse in cofactor form (row-major J[i][j]).
double det3(const double J[3][3]);
void inv3(const double J[3][3], double I[3][3]);
// Jacobian of tet (v0,v1,v2,v3): columns X1-X0, X2-X0, X3-X0.
void tet_jacobian(const Mesh& m, const std::array<int32_t, 4>& t, double J[3][3]);

// ASCII OpenFOAM constant/polyMesh (triangular faces, tetrahedral cells).
Mesh read_polymesh(const std::string& dir);
// Gmsh MSH 2.2 ASCII: tetrahedra (type 4) and tagged boundary triangles
// (type 2); physical tag 1 = inlet, 2 = outlet, 3 = wall.
Mesh read_msh2(const std::string& path);
// Binary HXT1 ("HXT1BIN1", version 1): the mixed hex/tet mesh format of the
// reference's hybrid and SST solvers (gpu/serial_cuda/hybrid_hxt1/
// hxt1_mesh.hpp:19-103).  Files without hex cells only: points, tets, and the
// inlet/outlet tet boundary records; every other exterior face is wall.
Mesh read_hxt1(const std::string& path);
// Raw arrays: points, tets (any orientation), boundary triangles with a patch
// index into patch_names.
Mesh mesh_from_arrays(int np, const double* xyz, int nc, const int32_t* tets, int nb,
                      const int32_t* btri, const int32_t* bpatch,
                      const std::vector<std::string>& patch_names);

// Patch order used when a mesh is built from cells: wall, inlet, outlet.
extern const char* const kCanonicalPatches[3];

}  // namespace nds
