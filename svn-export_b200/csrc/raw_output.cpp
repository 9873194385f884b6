// The flow field text output of DarcyFlowMHOutput::output_internal_flow_data
// (src/flow/darcy_flow_mh_output.cc:793-829): one "$FlowField" block per output time, each
// element on one line with its id, pressure, the flux vector at its centre, its number of sides,
// the pressures on its sides (the edge pressures of the sides' edges) and its side fluxes.
// Numbers are printed with "%.8g " exactly as the reference does, so files can be compared with
// the reference's raw_output.txt line by line.  Host code only: it reads host arrays that the
// caller fetched with mh_get_solution, mh_get_element_flux and mh_get_topology.
#include <cstdio>

#include "mh_darcy.h"

extern "C" int mh_raw_output_write(const char *path, int append, double time, int64_t n_el, const int32_t *el_id,
                                   const int32_t *el_side_start, const int32_t *side_edge, const double *solution,
                                   const double *el_flux) {
    if (!path || n_el < 0 || !el_side_start || !side_edge || !solution || !el_flux) return MH_ERR_INVALID;
    FILE *f = std::fopen(path, append ? "a" : "w");
    if (!f) return MH_ERR_INVALID;
    // the MH solution layout: [side fluxes | element pressures | edge pressures]
    const int64_t n_sides = el_side_start[n_el];
    const double *pressure = solution + n_sides, *edge_p = solution + n_sides + n_el;
    std::fprintf(f, "// fields:\n//ele_id    ele_presure    flux_in_barycenter[3]    n_sides   "
                    "side_pressures[n]    side_fluxes[n]\n");
    std::fprintf(f, "$FlowField\nT=");
    std::fprintf(f, "%.8g ", time);
    std::fprintf(f, "\n%lld\n", (long long)n_el);
    for (int64_t e = 0; e < n_el; ++e) {
        std::fprintf(f, "%d ", el_id ? el_id[e] : (int)e);
        std::fprintf(f, "%.8g ", pressure[e]);
        for (int k = 0; k < 3; ++k) std::fprintf(f, "%.8g ", el_flux[3 * e + k]);
        const int32_t s0 = el_side_start[e], ns = el_side_start[e + 1] - s0;
        std::fprintf(f, " %d ", ns);
        for (int32_t i = 0; i < ns; ++i) std::fprintf(f, "%.8g ", edge_p[side_edge[s0 + i]]);
        for (int32_t i = 0; i < ns; ++i) std::fprintf(f, "%.8g ", solution[s0 + i]);
        std::fprintf(f, "\n");
    }
    std::fprintf(f, "$EndFlowField\n\n");
    const int bad = std::ferror(f);
    return (std::fclose(f) != 0 || bad) ? MH_ERR_INVALID : MH_OK;
}
