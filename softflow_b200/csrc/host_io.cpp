// host_io.cpp -- VTK output of a channel's state, written on the host from
// the device state (pulled once per call through the state-transfer entry
// points).  The files have the layout and number formatting of the
// reference's VTKWriter (src/io/vtk_writer.cpp), so ParaView pipelines and
// scripts written for the reference read them unchanged.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/softflow_gpu.h"

namespace sfg_host {
void set_error(const std::string& msg);
}

namespace {

int io_fail(const char* path) {
    sfg_host::set_error(std::string("cannot open ") + path + " for writing");
    return SFG_ERR_ARG;
}

struct FieldData {
    int nx = 0, ny = 0;
    bool periodic_y = false, scalar = false;
    std::vector<double> rho, ux, uy, Fx, Fy, C;
};

int pull_field(sfg_context* ctx, int ch, bool want_force, bool want_c, FieldData& d) {
    sfg_channel_params p;
    int rc = sfg_get_channel_params(ctx, ch, &p);
    if (rc) return rc;
    d.nx = p.nx;
    d.ny = p.ny;
    d.periodic_y = p.periodic_y != 0;
    d.scalar = p.scalar_enabled != 0;
    const size_t N = (size_t)p.nx * p.ny;
    d.rho.resize(N);
    d.ux.resize(N);
    d.uy.resize(N);
    if (want_force) {
        d.Fx.resize(N);
        d.Fy.resize(N);
    }
    rc = sfg_get_macroscopic(ctx, ch, d.rho.data(), d.ux.data(), d.uy.data(),
                             want_force ? d.Fx.data() : nullptr,
                             want_force ? d.Fy.data() : nullptr);
    if (rc) return rc;
    if (want_c && d.scalar) {
        d.C.resize(N);
        rc = sfg_get_concentration(ctx, ch, d.C.data(), nullptr);
        if (rc) return rc;
    }
    return SFG_OK;
}

// CellType of the channel: SOLID (1) rows 0 and ny-1 unless periodic in y,
// FLUID (0) elsewhere (reference core/types.h:48-56).
inline int cell_type(const FieldData& d, int y) {
    return (!d.periodic_y && (y == 0 || y == d.ny - 1)) ? 1 : 0;
}

// Central differences with clamped neighbours (vtk_writer.cpp:39-73).
double vorticity(const FieldData& d, int x, int y) {
    const int xp = std::min(x + 1, d.nx - 1), xm = std::max(x - 1, 0);
    const int yp = std::min(y + 1, d.ny - 1), ym = std::max(y - 1, 0);
    const double duy_dx = (d.uy[(size_t)y * d.nx + xp] - d.uy[(size_t)y * d.nx + xm]) / (double)(xp - xm);
    const double dux_dy = (d.ux[(size_t)yp * d.nx + x] - d.ux[(size_t)ym * d.nx + x]) / (double)(yp - ym);
    return duy_dx - dux_dy;
}

double strain_rate(const FieldData& d, int x, int y) {
    const int xp = std::min(x + 1, d.nx - 1), xm = std::max(x - 1, 0);
    const int yp = std::min(y + 1, d.ny - 1), ym = std::max(y - 1, 0);
    const double dux_dx = (d.ux[(size_t)y * d.nx + xp] - d.ux[(size_t)y * d.nx + xm]) / (double)(xp - xm);
    const double duy_dy = (d.uy[(size_t)yp * d.nx + x] - d.uy[(size_t)ym * d.nx + x]) / (double)(yp - ym);
    const double dux_dy = (d.ux[(size_t)yp * d.nx + x] - d.ux[(size_t)ym * d.nx + x]) / (double)(yp - ym);
    const double duy_dx = (d.uy[(size_t)y * d.nx + xp] - d.uy[(size_t)y * d.nx + xm]) / (double)(xp - xm);
    const double s11 = dux_dx, s22 = duy_dy, s12 = 0.5 * (dux_dy + duy_dx);
    return std::sqrt(2.0 * (s11 * s11 + s22 * s22 + 2.0 * s12 * s12));
}

// One fluid array: the XML DataArray or the legacy SCALARS / VECTORS block.
struct Writer {
    FILE* fp;
    bool legacy;
    void begin_scalar(const char* name, const char* xml_type, const char* legacy_type) {
        if (legacy) {
            std::fprintf(fp, "SCALARS %s %s 1\n", name, legacy_type);
            std::fprintf(fp, "LOOKUP_TABLE default\n");
        } else {
            std::fprintf(fp, "<DataArray type=\"%s\" Name=\"%s\" format=\"ascii\">\n", xml_type, name);
        }
    }
    void begin_vector(const char* name) {
        if (legacy)
            std::fprintf(fp, "VECTORS %s double\n", name);
        else
            std::fprintf(fp, "<DataArray type=\"Float64\" Name=\"%s\" NumberOfComponents=\"3\" format=\"ascii\">\n",
                         name);
    }
    void end() {
        if (!legacy) std::fprintf(fp, "</DataArray>\n");
    }
};

struct PolyCopy {
    int capsule;
    std::vector<double> x, y;
};

}  // namespace

extern "C" int sfg_write_vtk_fluid(sfg_context* ctx, int channel, const char* output_dir, int step,
                                   int legacy, unsigned fields) {
    if (!ctx || !output_dir) {
        sfg_host::set_error("sfg_write_vtk_fluid: null argument");
        return SFG_ERR_ARG;
    }
    FieldData d;
    const bool want_c = (fields & SFG_VTK_CONCENTRATION) != 0;
    int rc = pull_field(ctx, channel, (fields & SFG_VTK_IBM_FORCE) != 0, want_c, d);
    if (rc) return rc;
    const std::string dir(output_dir);
    ::mkdir(dir.c_str(), 0755);
    char fn[1024];
    if (legacy) {
        std::snprintf(fn, sizeof(fn), "%s/fluid_%06d.vtk", dir.c_str(), step);
    } else {
        ::mkdir((dir + "/fluid").c_str(), 0755);
        ::mkdir((dir + "/particles").c_str(), 0755);
        std::snprintf(fn, sizeof(fn), "%s/fluid/fluid_%06d.vti", dir.c_str(), step);
    }
    FILE* fp = std::fopen(fn, "w");
    if (!fp) return io_fail(fn);
    const int nx = d.nx, ny = d.ny;
    Writer w{fp, legacy != 0};
    if (legacy) {
        std::fprintf(fp, "# vtk DataFile Version 3.0\n");
        std::fprintf(fp, "SoftFlow fluid field step %d\n", step);
        std::fprintf(fp, "ASCII\n");
        std::fprintf(fp, "DATASET STRUCTURED_POINTS\n");
        std::fprintf(fp, "DIMENSIONS %d %d 1\n", nx, ny);
        std::fprintf(fp, "ORIGIN 0 0 0\n");
        std::fprintf(fp, "SPACING 1 1 1\n");
        std::fprintf(fp, "POINT_DATA %d\n", nx * ny);
    } else {
        std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
        std::fprintf(fp, "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\">\n");
        std::fprintf(fp, "<ImageData WholeExtent=\"0 %d 0 %d 0 0\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n",
                     nx - 1, ny - 1);
        std::fprintf(fp, "<Piece Extent=\"0 %d 0 %d 0 0\">\n", nx - 1, ny - 1);
        std::fprintf(fp, "<PointData Scalars=\"density\" Vectors=\"velocity\">\n");
    }
    const size_t N = (size_t)nx * ny;
    if (fields & SFG_VTK_DENSITY) {
        w.begin_scalar("density", "Float64", "double");
        for (size_t i = 0; i < N; ++i) std::fprintf(fp, "%.6e\n", d.rho[i]);
        w.end();
    }
    if (fields & SFG_VTK_VELOCITY) {
        w.begin_vector("velocity");
        for (size_t i = 0; i < N; ++i) std::fprintf(fp, "%.6e %.6e 0\n", d.ux[i], d.uy[i]);
        w.end();
    }
    if (fields & SFG_VTK_VELOCITY_MAG) {
        w.begin_scalar("velocity_magnitude", "Float64", "double");
        for (size_t i = 0; i < N; ++i) std::fprintf(fp, "%.6e\n", std::sqrt(d.ux[i] * d.ux[i] + d.uy[i] * d.uy[i]));
        w.end();
    }
    if (fields & SFG_VTK_PRESSURE) {
        w.begin_scalar("pressure", "Float64", "double");
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x)
                std::fprintf(fp, "%.6e\n", cell_type(d, y) == 0 ? d.rho[(size_t)y * nx + x] / 3.0 : 0.0);
        w.end();
        w.begin_scalar("pressure_fluctuation", "Float64", "double");
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x)
                std::fprintf(fp, "%.6e\n",
                             cell_type(d, y) == 0 ? (d.rho[(size_t)y * nx + x] - 1.0) / 3.0 : 0.0);
        w.end();
    }
    if (fields & SFG_VTK_VORTICITY) {
        w.begin_scalar("vorticity", "Float64", "double");
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) std::fprintf(fp, "%.6e\n", vorticity(d, x, y));
        w.end();
    }
    if (fields & SFG_VTK_STRAIN_RATE) {
        w.begin_scalar("strain_rate", "Float64", "double");
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) std::fprintf(fp, "%.6e\n", strain_rate(d, x, y));
        w.end();
    }
    if (fields & SFG_VTK_IBM_FORCE) {
        w.begin_vector("ibm_force");
        for (size_t i = 0; i < N; ++i) std::fprintf(fp, "%.6e %.6e 0\n", d.Fx[i], d.Fy[i]);
        w.end();
    }
    if (fields & SFG_VTK_NODE_TYPE) {
        w.begin_scalar("node_type", "Int32", "int");
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) std::fprintf(fp, "%d\n", cell_type(d, y));
        w.end();
    }
    if (want_c && d.scalar) {
        w.begin_scalar("concentration", "Float64", "double");
        for (size_t i = 0; i < N; ++i) std::fprintf(fp, "%.6e\n", d.C[i]);
        w.end();
    }
    if (!legacy) {
        std::fprintf(fp, "</PointData>\n");
        std::fprintf(fp, "</Piece>\n</ImageData>\n</VTKFile>\n");
    }
    std::fflush(fp);
    std::fclose(fp);
    return SFG_OK;
}

extern "C" int sfg_write_vtk_capsules(sfg_context* ctx, int channel, const char* output_dir,
                                      int step, int legacy, const int* type_ids) {
    if (!ctx || !output_dir) {
        sfg_host::set_error("sfg_write_vtk_capsules: null argument");
        return SFG_ERR_ARG;
    }
    int ncaps = 0, M = 0;
    int rc = sfg_channel_counts(ctx, channel, &ncaps, &M);
    if (rc) return rc;
    if (ncaps == 0) return SFG_OK;
    sfg_channel_params p;
    if ((rc = sfg_get_channel_params(ctx, channel, &p))) return rc;
    std::vector<int> nodes(ncaps);
    if ((rc = sfg_get_capsule_nodes(ctx, channel, nodes.data()))) return rc;
    std::vector<double> pos(2 * (size_t)M), vel(2 * (size_t)M), frc(2 * (size_t)M);
    if ((rc = sfg_get_markers(ctx, channel, pos.data(), vel.data(), frc.data()))) return rc;
    // deformation index of every capsule (device reduction, reference order)
    int nch = 0, base = 0;
    if ((rc = sfg_num_channels(ctx, &nch))) return rc;
    if ((rc = sfg_get_capsule_base(ctx, channel, &base))) return rc;
    int total = 0;
    for (int c = 0; c < nch; ++c) {
        int k = 0;
        if ((rc = sfg_channel_counts(ctx, c, &k, nullptr))) return rc;
        total += k;
    }
    std::vector<sfg_capsule_stats> st((size_t)std::max(total, 1));
    if ((rc = sfg_thermo(ctx, nullptr, st.data()))) return rc;
    std::vector<int> off(ncaps + 1, 0);
    for (int c = 0; c < ncaps; ++c) off[c + 1] = off[c] + nodes[c];

    const std::string dir(output_dir);
    ::mkdir(dir.c_str(), 0755);
    char fn[1024];
    if (legacy) {
        std::snprintf(fn, sizeof(fn), "%s/particles_%06d.vtk", dir.c_str(), step);
    } else {
        ::mkdir((dir + "/fluid").c_str(), 0755);
        ::mkdir((dir + "/particles").c_str(), 0755);
        std::snprintf(fn, sizeof(fn), "%s/particles/particles_%06d.vtp", dir.c_str(), step);
    }
    // The reference's capsules are periodic in x for periodic channels
    // (VTKWriter::setPeriodicX); every channel here is.
    const double Lx = (double)p.nx;
    std::vector<PolyCopy> copies;
    copies.reserve(2 * (size_t)ncaps);
    for (int c = 0; c < ncaps; ++c) {
        const int n = nodes[c];
        const double* X = pos.data() + 2 * (size_t)off[c];
        // unwrapNodes (vtk_writer.cpp:211-228)
        std::vector<double> ux(n), uy(n);
        ux[0] = X[0];
        uy[0] = X[1];
        for (int k = 1; k < n; ++k) {
            double dx = X[2 * k] - X[2 * (k - 1)];
            const double dy = X[2 * k + 1] - X[2 * (k - 1) + 1];
            if (dx > 0.5 * Lx) dx -= Lx;
            if (dx < -0.5 * Lx) dx += Lx;
            ux[k] = ux[k - 1] + dx;
            uy[k] = uy[k - 1] + dy;
        }
        double xmin = ux[0], xmax = ux[0];
        for (int k = 0; k < n; ++k) {
            if (ux[k] < xmin) xmin = ux[k];
            if (ux[k] > xmax) xmax = ux[k];
        }
        const bool exits_right = xmax >= Lx, exits_left = xmin < 0.0;
        if (!exits_right && !exits_left) {
            copies.push_back({c, ux, uy});
        } else {
            PolyCopy a{c, std::vector<double>(n), uy}, b{c, std::vector<double>(n), uy};
            const double shift = exits_right ? -Lx : Lx;
            for (int k = 0; k < n; ++k) {
                a.x[k] = std::clamp(ux[k], 0.0, Lx);
                b.x[k] = std::clamp(ux[k] + shift, 0.0, Lx);
            }
            copies.push_back(std::move(a));
            copies.push_back(std::move(b));
        }
    }
    int total_nodes = 0;
    const int total_polys = (int)copies.size();
    for (const auto& cp : copies) total_nodes += (int)cp.x.size();
    auto tid = [&](int c) { return type_ids ? type_ids[c] : 0; };
    FILE* fp = std::fopen(fn, "w");
    if (!fp) return io_fail(fn);
    const bool scalar = p.scalar_enabled != 0;
    if (legacy) {
        std::fprintf(fp, "# vtk DataFile Version 3.0\n");
        std::fprintf(fp, "SoftFlow particles step %d\n", step);
        std::fprintf(fp, "ASCII\n");
        std::fprintf(fp, "DATASET POLYDATA\n");
        std::fprintf(fp, "POINTS %d double\n", total_nodes);
        for (const auto& cp : copies)
            for (size_t k = 0; k < cp.x.size(); ++k) std::fprintf(fp, "%.6e %.6e 0\n", cp.x[k], cp.y[k]);
        std::fprintf(fp, "POLYGONS %d %d\n", total_polys, total_polys + total_nodes);
        int o = 0;
        for (const auto& cp : copies) {
            const int nn = (int)cp.x.size();
            std::fprintf(fp, "%d", nn);
            for (int k = 0; k < nn; ++k) std::fprintf(fp, " %d", o + k);
            std::fprintf(fp, "\n");
            o += nn;
        }
        std::fprintf(fp, "POINT_DATA %d\n", total_nodes);
        std::fprintf(fp, "SCALARS capsule_id int 1\n");
        std::fprintf(fp, "LOOKUP_TABLE default\n");
        for (const auto& cp : copies)
            for (size_t k = 0; k < cp.x.size(); ++k) std::fprintf(fp, "%d\n", cp.capsule);
        std::fprintf(fp, "SCALARS capsule_type int 1\n");
        std::fprintf(fp, "LOOKUP_TABLE default\n");
        for (const auto& cp : copies)
            for (size_t k = 0; k < cp.x.size(); ++k) std::fprintf(fp, "%d\n", tid(cp.capsule));
        std::fprintf(fp, "VECTORS node_velocity double\n");
        for (const auto& cp : copies)
            for (int k = off[cp.capsule]; k < off[cp.capsule + 1]; ++k)
                std::fprintf(fp, "%.6e %.6e 0\n", vel[2 * (size_t)k], vel[2 * (size_t)k + 1]);
        std::fprintf(fp, "VECTORS node_force double\n");
        for (const auto& cp : copies)
            for (int k = off[cp.capsule]; k < off[cp.capsule + 1]; ++k)
                std::fprintf(fp, "%.6e %.6e 0\n", frc[2 * (size_t)k], frc[2 * (size_t)k + 1]);
        if (scalar) {
            std::fprintf(fp, "SCALARS gamma double 1\n");
            std::fprintf(fp, "LOOKUP_TABLE default\n");
            for (const auto& cp : copies)
                for (int k = off[cp.capsule]; k < off[cp.capsule + 1]; ++k) std::fprintf(fp, "%.6e\n", 0.0);
        }
        // per-polygon quantities (vtk_writer.cpp:821-913)
        std::fprintf(fp, "CELL_DATA %d\n", total_polys);
        std::fprintf(fp, "SCALARS capsule_id_cell int 1\n");
        std::fprintf(fp, "LOOKUP_TABLE default\n");
        for (const auto& cp : copies) std::fprintf(fp, "%d\n", cp.capsule);
        std::fprintf(fp, "SCALARS cell_type int 1\n");
        std::fprintf(fp, "LOOKUP_TABLE default\n");
        for (const auto& cp : copies) std::fprintf(fp, "%d\n", tid(cp.capsule));
        std::fprintf(fp, "SCALARS deformation_index double 1\n");
        std::fprintf(fp, "LOOKUP_TABLE default\n");
        for (const auto& cp : copies) std::fprintf(fp, "%.6e\n", st[(size_t)base + cp.capsule].deformation);
        std::vector<double> avx(ncaps), avy(ncaps), ftx(ncaps), fty(ncaps);
        for (int c = 0; c < ncaps; ++c) {
            double ax = 0.0, ay = 0.0, fx = 0.0, fy = 0.0;
            for (int k = off[c]; k < off[c + 1]; ++k) {
                ax += vel[2 * (size_t)k];
                ay += vel[2 * (size_t)k + 1];
                fx += frc[2 * (size_t)k];
                fy += frc[2 * (size_t)k + 1];
            }
            avx[c] = ax / nodes[c];
            avy[c] = ay / nodes[c];
            ftx[c] = fx;
            fty[c] = fy;
        }
        std::fprintf(fp, "VECTORS particle_velocity double\n");
        for (const auto& cp : copies) std::fprintf(fp, "%.6e %.6e 0\n", avx[cp.capsule], avy[cp.capsule]);
        std::fprintf(fp, "VECTORS particle_force double\n");
        for (const auto& cp : copies) std::fprintf(fp, "%.6e %.6e 0\n", ftx[cp.capsule], fty[cp.capsule]);
        std::fprintf(fp, "SCALARS particle_speed double 1\n");
        std::fprintf(fp, "LOOKUP_TABLE default\n");
        for (const auto& cp : copies) {
            const double ax = avx[cp.capsule], ay = avy[cp.capsule];
            std::fprintf(fp, "%.6e\n", std::sqrt(ax * ax + ay * ay));
        }
        std::fprintf(fp, "SCALARS particle_area double 1\n");
        std::fprintf(fp, "LOOKUP_TABLE default\n");
        for (const auto& cp : copies) std::fprintf(fp, "%.6e\n", st[(size_t)base + cp.capsule].area);
        std::fprintf(fp, "SCALARS particle_perimeter double 1\n");
        std::fprintf(fp, "LOOKUP_TABLE default\n");
        for (const auto& cp : copies) std::fprintf(fp, "%.6e\n", st[(size_t)base + cp.capsule].perimeter);
        if (scalar) {
            // no capsule chemistry on this path: nothing released or
            // absorbed, infinite reservoirs (-1), no surface coverage
            const char* names[4] = {"scalar_released", "scalar_absorbed", "Mp", "gamma_mean"};
            const double vals[4] = {0.0, 0.0, -1.0, 0.0};
            for (int a = 0; a < 4; ++a) {
                std::fprintf(fp, "SCALARS %s double 1\n", names[a]);
                std::fprintf(fp, "LOOKUP_TABLE default\n");
                for (size_t k = 0; k < copies.size(); ++k) std::fprintf(fp, "%.6e\n", vals[a]);
            }
        }
        std::fflush(fp);
        std::fclose(fp);
        return SFG_OK;
    }
    std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
    std::fprintf(fp, "<VTKFile type=\"PolyData\" version=\"1.0\" byte_order=\"LittleEndian\">\n");
    std::fprintf(fp, "<PolyData>\n");
    std::fprintf(fp, "<Piece NumberOfPoints=\"%d\" NumberOfVerts=\"0\" NumberOfLines=\"0\" "
                     "NumberOfStrips=\"0\" NumberOfPolys=\"%d\">\n",
                 total_nodes, total_polys);
    std::fprintf(fp, "<Points>\n");
    std::fprintf(fp, "<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (const auto& cp : copies)
        for (size_t k = 0; k < cp.x.size(); ++k) std::fprintf(fp, "%.6e %.6e 0\n", cp.x[k], cp.y[k]);
    std::fprintf(fp, "</DataArray>\n</Points>\n");
    std::fprintf(fp, "<Polys>\n");
    std::fprintf(fp, "<DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n");
    int o = 0;
    for (const auto& cp : copies) {
        const int nn = (int)cp.x.size();
        for (int k = 0; k < nn; ++k) std::fprintf(fp, "%d ", o + k);
        std::fprintf(fp, "\n");
        o += nn;
    }
    std::fprintf(fp, "</DataArray>\n");
    std::fprintf(fp, "<DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n");
    o = 0;
    for (const auto& cp : copies) {
        o += (int)cp.x.size();
        std::fprintf(fp, "%d ", o);
    }
    std::fprintf(fp, "\n</DataArray>\n");
    std::fprintf(fp, "</Polys>\n");
    std::fprintf(fp, "<PointData>\n");
    std::fprintf(fp, "<DataArray type=\"Int32\" Name=\"capsule_id\" format=\"ascii\">\n");
    for (const auto& cp : copies)
        for (size_t k = 0; k < cp.x.size(); ++k) std::fprintf(fp, "%d ", cp.capsule);
    std::fprintf(fp, "\n</DataArray>\n");
    std::fprintf(fp, "<DataArray type=\"Int32\" Name=\"capsule_type\" format=\"ascii\">\n");
    for (const auto& cp : copies)
        for (size_t k = 0; k < cp.x.size(); ++k) std::fprintf(fp, "%d ", tid(cp.capsule));
    std::fprintf(fp, "\n</DataArray>\n");
    std::fprintf(fp, "<DataArray type=\"Float64\" Name=\"velocity\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (const auto& cp : copies)
        for (int k = off[cp.capsule]; k < off[cp.capsule + 1]; ++k)
            std::fprintf(fp, "%.6e %.6e 0\n", vel[2 * (size_t)k], vel[2 * (size_t)k + 1]);
    std::fprintf(fp, "</DataArray>\n");
    std::fprintf(fp, "<DataArray type=\"Float64\" Name=\"force\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (const auto& cp : copies)
        for (int k = off[cp.capsule]; k < off[cp.capsule + 1]; ++k)
            std::fprintf(fp, "%.6e %.6e 0\n", frc[2 * (size_t)k], frc[2 * (size_t)k + 1]);
    std::fprintf(fp, "</DataArray>\n");
    if (scalar) {
        std::fprintf(fp, "<DataArray type=\"Float64\" Name=\"gamma\" format=\"ascii\">\n");
        for (const auto& cp : copies)
            for (int k = off[cp.capsule]; k < off[cp.capsule + 1]; ++k) std::fprintf(fp, "%.6e\n", 0.0);
        std::fprintf(fp, "</DataArray>\n");
    }
    std::fprintf(fp, "</PointData>\n");
    std::fprintf(fp, "<CellData>\n");
    std::fprintf(fp, "<DataArray type=\"Int32\" Name=\"cell_capsule_id\" format=\"ascii\">\n");
    for (const auto& cp : copies) std::fprintf(fp, "%d ", cp.capsule);
    std::fprintf(fp, "\n</DataArray>\n");
    std::fprintf(fp, "<DataArray type=\"Int32\" Name=\"cell_capsule_type\" format=\"ascii\">\n");
    for (const auto& cp : copies) std::fprintf(fp, "%d ", tid(cp.capsule));
    std::fprintf(fp, "\n</DataArray>\n");
    std::fprintf(fp, "<DataArray type=\"Float64\" Name=\"deformation_index\" format=\"ascii\">\n");
    for (const auto& cp : copies) std::fprintf(fp, "%.6e ", st[(size_t)base + cp.capsule].deformation);
    std::fprintf(fp, "\n</DataArray>\n");
    std::fprintf(fp, "<DataArray type=\"Float64\" Name=\"capsule_speed\" format=\"ascii\">\n");
    for (const auto& cp : copies) {
        const int n = nodes[cp.capsule];
        double ax = 0.0, ay = 0.0;
        for (int k = off[cp.capsule]; k < off[cp.capsule + 1]; ++k) {
            ax += vel[2 * (size_t)k];
            ay += vel[2 * (size_t)k + 1];
        }
        ax /= n;
        ay /= n;
        std::fprintf(fp, "%.6e ", std::sqrt(ax * ax + ay * ay));
    }
    std::fprintf(fp, "\n</DataArray>\n");
    if (scalar) {
        // no capsule chemistry on this path: infinite reservoirs (-1), no
        // surface coverage, nothing released or absorbed
        const char* names[4] = {"Mp", "gamma_mean", "cumulative_released", "cumulative_absorbed"};
        const double vals[4] = {-1.0, 0.0, 0.0, 0.0};
        for (int a = 0; a < 4; ++a) {
            std::fprintf(fp, "<DataArray type=\"Float64\" Name=\"%s\" format=\"ascii\">\n", names[a]);
            for (size_t k = 0; k < copies.size(); ++k) std::fprintf(fp, "%.6e ", vals[a]);
            std::fprintf(fp, "\n</DataArray>\n");
        }
    }
    std::fprintf(fp, "</CellData>\n");
    std::fprintf(fp, "</Piece>\n</PolyData>\n</VTKFile>\n");
    std::fflush(fp);
    std::fclose(fp);
    return SFG_OK;
}
