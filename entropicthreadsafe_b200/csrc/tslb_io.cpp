// tslb_io.cpp -- the print_module.f90 file formats (include/tslb_io.h).
// Host code only: the writers take host arrays and need no GPU.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/tslb_io.h"

namespace {

// right-aligned in `width` characters (space_fmtnumb / space_fmtnumb12)
std::string padded(long long v, int width, char fill) {
    std::string s = std::to_string(v);
    if ((int)s.size() < width) s = std::string(width - s.size(), fill) + s;
    return s;
}

bool write_all(FILE* f, const void* p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }

// VTK ImageData header in the segment layout of header_vtk: every line has
// a fixed length because the extents are 6-character fields and the offset a
// 12-character field.
std::string vti_header(int nx, int ny, int nz, const std::string& name8, int ncomp) {
    const std::string ext = padded(1, 6, ' ') + " " + padded(nx, 6, ' ') + " " + padded(1, 6, ' ') + " " +
                            padded(ny, 6, ' ') + " " + padded(1, 6, ' ') + " " + padded(nz, 6, ' ');
    std::string h;
    h += "<?xml version=\"1.0\"?>\n";
    h += "<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    h += "  <ImageData WholeExtent=\"" + ext + "\">\n";
    h += "    <Piece Extent=\"" + ext + "\">\n";
    h += "      <PointData>\n";
    h += "        <DataArray type=\"Float32\" Name=\"" + name8 + "\" NumberOfComponents=\"" + std::to_string(ncomp) +
         "\" format=\"appended\" offset=\"" + padded(0, 12, ' ') + "\"/>\n";
    h += "      </PointData>\n";
    h += "    </Piece>\n";
    h += "  </ImageData>\n";
    h += "  <AppendedData encoding=\"raw\">\n";
    h += "_";
    return h;
}

const char kVtiFooter[] = "\n  </AppendedData>\n</VTKFile>\n";

}  // namespace

extern "C" {

int tslb_frame_path(char* out, int cap, const char* dir, const char* prefix, const char* name, int frame,
                    const char* ext) {
    if (!out || cap <= 0 || !dir || !prefix || !name || !ext || frame < 0) return TSLB_ERR_ARG;
    std::string d(dir);
    if (!d.empty() && d.back() != '/') d += '/';
    const std::string p = d + prefix + "_" + name + "_" + padded(frame, 6, '0') + "." + ext;
    if ((int)p.size() + 1 > cap) return TSLB_ERR_ARG;
    std::memcpy(out, p.c_str(), p.size() + 1);
    return TSLB_OK;
}

int tslb_write_raw(const char* path, const float* data, long long n) {
    if (!path || n < 0 || (n > 0 && !data)) return TSLB_ERR_ARG;
    FILE* f = std::fopen(path, "wb");
    if (!f) return TSLB_ERR_ARG;
    const bool ok = write_all(f, data, sizeof(float) * (size_t)n);
    return (std::fclose(f) == 0 && ok) ? TSLB_OK : TSLB_ERR_ARG;
}

int tslb_write_vti(const char* path, const char* name, int nx, int ny, int nz, int ncomp, const float* data) {
    if (!path || !name || nx < 1 || ny < 1 || nz < 1 || (ncomp != 1 && ncomp != 3) || !data) return TSLB_ERR_ARG;
    std::string name8(name);
    if (name8.size() > 8) return TSLB_ERR_ARG;
    name8.resize(8, ' ');
    const long long n = (long long)nx * ny * nz * ncomp;
    if (n * 4 > INT32_MAX) return TSLB_ERR_ARG;   // the byte count is an int32, as in the reference
    const int32_t nbytes = (int32_t)(n * 4);
    const std::string head = vti_header(nx, ny, nz, name8, ncomp);
    FILE* f = std::fopen(path, "wb");
    if (!f) return TSLB_ERR_ARG;
    bool ok = write_all(f, head.data(), head.size());
    ok = ok && write_all(f, &nbytes, sizeof(nbytes));
    ok = ok && write_all(f, data, (size_t)nbytes);
    ok = ok && write_all(f, kVtiFooter, sizeof(kVtiFooter) - 1);
    return (std::fclose(f) == 0 && ok) ? TSLB_OK : TSLB_ERR_ARG;
}

int tslb_write_slices(const char* dir, const char* name, int frame, int nx, int ny, int nz, const float* field) {
    if (!dir || !name || nx < 2 || ny < 2 || nz < 2 || !field || frame < 0) return TSLB_ERR_ARG;
    // 1-based nx/2 etc. of the reference -> 0-based index nx/2 - 1
    const int xm = nx / 2 - 1, ym = ny / 2 - 1, zm = nz / 2 - 1;
    auto at = [&](int x, int y, int z) { return field[x + (size_t)nx * (y + (size_t)ny * z)]; };
    const char* tags[3] = {"xy", "xz", "yz"};
    for (int t = 0; t < 3; ++t) {
        std::string buf;
        std::string tag = std::string(name) + tags[t];
        char path[4096];
        if (tslb_frame_path(path, sizeof(path), dir, "out", tag.c_str(), frame, "raw")) return TSLB_ERR_ARG;
        std::string bytes;
        if (t == 0) {
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) { float v = at(x, y, zm); bytes.append((const char*)&v, 4); }
        } else if (t == 1) {
            for (int z = 0; z < nz; ++z)
                for (int x = 0; x < nx; ++x) { float v = at(x, ym, z); bytes.append((const char*)&v, 4); }
        } else {
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y) { float v = at(xm, y, z); bytes.append((const char*)&v, 4); }
        }
        FILE* f = std::fopen(path, "wb");
        if (!f) return TSLB_ERR_ARG;
        const bool ok = write_all(f, bytes.data(), bytes.size());
        if (std::fclose(f) != 0 || !ok) return TSLB_ERR_ARG;
    }
    return TSLB_OK;
}

}  // extern "C"
