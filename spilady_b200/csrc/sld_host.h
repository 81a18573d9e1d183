// Host-side geometry: box, link cells, colour groups, the initial atom order.
#pragma once
#include <string>
#include <vector>

#include "../../include/sld.h"

namespace sld {

struct HostGeom {
    double d[6], inv[6], box_len[3], box_volume;
    double rcut_max, min_len;
    int nx, ny, nz, ncells;
    int tx, ty, tz, nte;
    int ngroups, te_ngroups;
    std::vector<int> gstart, gcells;        // link-cell colour groups
    std::vector<int> te_gstart, te_gcells;  // Te-cell colour groups
    // core_dTe's colour sweep as levels and the neighbour table of the Te
    // cells in colour order (te_levels); empty above 32,767 cells
    int te_nlevels = 0;
    std::vector<int> te_lstart;
    std::vector<unsigned short> te_ltasks, te_lnb;
};

// inverse box, edge lengths and volume from G.d (vec_utils_CPU.cpp:135-148,
// initial.cpp's box_length and box_volume)
void box_derived(HostGeom& G);

// Fills G from the parameters; id_of_slot / slot_of_id give the storage
// order (atoms sorted by initial link cell, each cell in the reference's
// initial list order).  r is not modified.
int setup_geometry(const sld_params& P, int natom, const std::vector<double>& r, HostGeom& G,
                   std::vector<int>& id_of_slot, std::vector<int>& slot_of_id);

// periodic_CPU.cpp:31-50 on the host
void host_periodic(const HostGeom& G, double& x, double& y, double& z);

// allocate_cells_CPU.cpp:33-125: greedy colouring of an nx*ny*nz periodic
// grid with the 26-neighbour stencil, cells scanned in index order
int colour_grid(int nx, int ny, int nz, std::vector<int>& gstart, std::vector<int>& gcells);

// The diffusion sweep of core_dTe's C step (core_dTe_CPU.cpp:140-175: colour
// groups 0..G-1, then G-1..0, on an nx*ny*nz periodic Te grid) as levels.
// An update reads its own cell and its six face neighbours, so it goes to
// the level after the latest level at which any of these was updated: every
// update then reads exactly the values of the sequential sweep, and a
// neighbour's later update lands on a later level.  A cell whose second
// update would follow its first one directly (no neighbour updated in
// between) is one task of two updates.
// Cells are named by their position in gcells (colour order), the order in
// which the sweep kernel stores them: tasks[] = position | 0x8000 for a
// double update, lstart[l]..lstart[l+1] are level l's tasks, and nbp holds
// 8 entries per position: the positions of the +x, -x, +y, -y, +z, -z
// neighbours, then 0, 0.  Returns the number of levels, or 0 (lists left
// empty) when a position does not fit 15 bits.
int te_levels(int nx, int ny, int nz, const std::vector<int>& gstart,
              const std::vector<int>& gcells, std::vector<int>& lstart,
              std::vector<unsigned short>& tasks, std::vector<unsigned short>& nbp);

// Output files in the reference's formats (sld_io.cpp).  out_path forms
// <dir>/<prefix><body>[_NNNN].dat (n_output < 0: no number); append_line adds
// "<step> v0 ... v(n-1)"; write_con_file writes a con- file (header, box,
// one row "<i> <element> ..." per atom of the natom x ncols table);
// write_cel_file a cel- file (one row per cell).
std::string out_path(const char* dir, const char* prefix, const char* body, int n_output);
int append_line(const std::string& path, int step, const double* v, int n);
int write_con_file(const std::string& path, long natom, double total_time, const double* box,
                   const char* type, const char* element, int ncols, const double* table);
int write_cel_file(const std::string& path, long ncells, double total_time, const double* box,
                   int ncols, const double* table);

}  // namespace sld
