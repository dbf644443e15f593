// Design-state files (host only).  They replace what the drivers do with
// MATLAB files and plots: the warm start from a saved design
// (CrossWalk/crosswalk.m:135 `load x46.mat`) and the isosurface plot at the
// end (display_3D), which here becomes a volume file for external viewers.
//
// Design state: a 64-byte little-endian header, then the parameters and the
// two element arrays as doubles in the solver's element order
// (e = nelz*nely*i + nely*k + j):
//   char magic[8] = "GPUTODS1"; uint32 version = 1; int32 nelx, nely, nelz;
//   int32 iteration; int32 nparams; uint32 narrays = 2; 28 reserved bytes
//   double params[nparams]; double x[nel]; double xPhys[nel]
// Volume export: a NRRD header (<base>.nhdr) and raw float32 data (<base>.raw),
// y fastest, then z, then x, as the element order stores them.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gputo.h"
#include "gputo_internal.h"

namespace {
struct DesignHeader {
    char magic[8];
    uint32_t version;
    int32_t nelx, nely, nelz, iteration, nparams;
    uint32_t narrays;
    char reserved[28];
};
static_assert(sizeof(DesignHeader) == 64, "design-state header is 64 bytes");
constexpr char kMagic[8] = {'G', 'P', 'U', 'T', 'O', 'D', 'S', '1'};

bool is_little_endian()
{
    const uint16_t v = 1;
    return *reinterpret_cast<const uint8_t *>(&v) == 1;
}
}  // namespace

extern "C" {

int gputo_design_save(const char *path, int nelx, int nely, int nelz, int iteration, const double *params,
                      int nparams, const double *x, const double *xPhys)
{
    if (!path || nelx < 1 || nely < 1 || nelz < 1 || nparams < 0 || (nparams > 0 && !params) || !x || !xPhys) {
        gputo::set_error("gputo_design_save: bad argument");
        return GPUTO_ERR_ARG;
    }
    if (!is_little_endian()) {
        gputo::set_error("gputo_design_save: big-endian hosts are not supported");
        return GPUTO_ERR_ARG;
    }
    DesignHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = 1;
    h.nelx = nelx, h.nely = nely, h.nelz = nelz, h.iteration = iteration, h.nparams = nparams;
    h.narrays = 2;
    const size_t nel = (size_t)nelx * nely * nelz;
    std::FILE *f = std::fopen(path, "wb");
    if (!f) {
        gputo::set_error(std::string("gputo_design_save: cannot open ") + path);
        return GPUTO_ERR_ARG;
    }
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    if (ok && nparams) ok = std::fwrite(params, sizeof(double), (size_t)nparams, f) == (size_t)nparams;
    if (ok) ok = std::fwrite(x, sizeof(double), nel, f) == nel;
    if (ok) ok = std::fwrite(xPhys, sizeof(double), nel, f) == nel;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        gputo::set_error(std::string("gputo_design_save: write failed for ") + path);
        return GPUTO_ERR_ARG;
    }
    return GPUTO_OK;
}

int gputo_design_load(const char *path, int *nelx, int *nely, int *nelz, int *iteration, double *params,
                      int *nparams, double *x, double *xPhys)
{
    if (!path || !nelx || !nely || !nelz || !nparams) {
        gputo::set_error("gputo_design_load: bad argument");
        return GPUTO_ERR_ARG;
    }
    std::FILE *f = std::fopen(path, "rb");
    if (!f) {
        gputo::set_error(std::string("gputo_design_load: cannot open ") + path);
        return GPUTO_ERR_ARG;
    }
    DesignHeader h{};
    auto fail = [&](const char *why) {
        std::fclose(f);
        gputo::set_error(std::string("gputo_design_load: ") + why + " (" + path + ")");
        return GPUTO_ERR_ARG;
    };
    if (std::fread(&h, sizeof(h), 1, f) != 1) return fail("file shorter than its header");
    if (std::memcmp(h.magic, kMagic, 8) != 0) return fail("not a design-state file");
    if (h.version != 1 || h.narrays != 2) return fail("unsupported design-state version");
    if (h.nelx < 1 || h.nely < 1 || h.nelz < 1 || h.nparams < 0) return fail("corrupt header");
    const int cap = *nparams;
    *nelx = h.nelx, *nely = h.nely, *nelz = h.nelz, *nparams = h.nparams;
    if (iteration) *iteration = h.iteration;
    if (!x && !xPhys && !params) {   // size query
        std::fclose(f);
        return GPUTO_OK;
    }
    if (params && cap < h.nparams) return fail("params buffer smaller than the saved parameter count");
    const size_t nel = (size_t)h.nelx * h.nely * h.nelz;
    std::vector<double> pbuf((size_t)h.nparams);
    if (h.nparams && std::fread(pbuf.data(), sizeof(double), pbuf.size(), f) != pbuf.size())
        return fail("truncated parameters");
    if (params && h.nparams) std::memcpy(params, pbuf.data(), sizeof(double) * pbuf.size());
    std::vector<double> tmp;
    double *dx = x;
    if (!dx) {
        tmp.resize(nel);
        dx = tmp.data();
    }
    if (std::fread(dx, sizeof(double), nel, f) != nel) return fail("truncated x");
    if (xPhys && std::fread(xPhys, sizeof(double), nel, f) != nel) return fail("truncated xPhys");
    std::fclose(f);
    return GPUTO_OK;
}

int gputo_design_export_volume(const char *base, int nelx, int nely, int nelz, const double *xPhys)
{
    if (!base || nelx < 1 || nely < 1 || nelz < 1 || !xPhys) {
        gputo::set_error("gputo_design_export_volume: bad argument");
        return GPUTO_ERR_ARG;
    }
    const std::string b(base), raw = b + ".raw", hdr = b + ".nhdr";
    const size_t nel = (size_t)nelx * nely * nelz;
    std::vector<float> v(nel);
    for (size_t e = 0; e < nel; ++e) v[e] = (float)xPhys[e];
    std::FILE *f = std::fopen(raw.c_str(), "wb");
    if (!f) {
        gputo::set_error("gputo_design_export_volume: cannot open " + raw);
        return GPUTO_ERR_ARG;
    }
    bool ok = std::fwrite(v.data(), sizeof(float), nel, f) == nel;
    ok = (std::fclose(f) == 0) && ok;
    const std::string leaf = raw.substr(raw.find_last_of('/') == std::string::npos ? 0 : raw.find_last_of('/') + 1);
    std::FILE *h = ok ? std::fopen(hdr.c_str(), "w") : nullptr;
    if (!h) {
        gputo::set_error("gputo_design_export_volume: cannot write " + (ok ? hdr : raw));
        return GPUTO_ERR_ARG;
    }
    std::fprintf(h,
                 "NRRD0004\n# xPhys of a gputo design, element order: y fastest, then z, then x\n"
                 "type: float\ndimension: 3\nsizes: %d %d %d\nspacings: 1 1 1\n"
                 "labels: \"y\" \"z\" \"x\"\nencoding: raw\nendian: little\ndata file: %s\n",
                 nely, nelz, nelx, leaf.c_str());
    ok = std::fclose(h) == 0;
    if (!ok) {
        gputo::set_error("gputo_design_export_volume: cannot write " + hdr);
        return GPUTO_ERR_ARG;
    }
    return GPUTO_OK;
}

}  // extern "C"
