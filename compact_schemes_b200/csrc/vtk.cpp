// vtk.cpp -- headless VTK writer (legacy format, binary big-endian floats), the
// layout of io::go_vtk (src/IO.hpp:108-159): a STRUCTURED_GRID whose point
// coordinates are the first three variables, then one SCALARS block per
// further variable.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "context.h"

namespace {

void put_be(std::vector<char> &buf, float v) {
    uint32_t u;
    std::memcpy(&u, &v, sizeof u);
    const char b[4] = {(char)(u >> 24), (char)(u >> 16), (char)(u >> 8), (char)u};
    buf.insert(buf.end(), b, b + 4);
}

}  // namespace

extern "C" int cs_vtk_write(const char *path, int lxi, int let, int lze, const float *data, int nvars,
                            const char *const *names) {
    using csb::set_error;
    if (!path || !data || lxi < 1 || let < 1 || lze < 1 || nvars < 3 || (nvars > 3 && !names))
        return set_error(CS_ERR_INVALID, "bad argument");
    const int64_t np = (int64_t)lxi * let * lze;
    std::vector<char> buf;
    char line[256];
    auto text = [&](const char *s) { buf.insert(buf.end(), s, s + std::strlen(s)); };
    text("# vtk DataFile Version 2.0\nOutput compact schemes\nBINARY\nDATASET STRUCTURED_GRID\n");
    std::snprintf(line, sizeof line, "DIMENSIONS %d %d %d\nPOINTS %lld float\n", lxi, let, lze, (long long)np);
    text(line);
    for (int64_t i = 0; i < np; ++i)
        for (int c = 0; c < 3; ++c) put_be(buf, data[c * np + i]);
    std::snprintf(line, sizeof line, "\nPOINT_DATA %lld\n", (long long)np);
    text(line);
    for (int v = 3; v < nvars; ++v) {
        if (!names[v - 3] || std::strlen(names[v - 3]) > 64) return set_error(CS_ERR_INVALID, "variable name");
        std::snprintf(line, sizeof line, "SCALARS %s float 1\nLOOKUP_TABLE default\n", names[v - 3]);
        text(line);
        for (int64_t i = 0; i < np; ++i) put_be(buf, data[v * np + i]);
        text("\n");
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return set_error(CS_ERR_INVALID, "cannot open %s", path);
    const size_t w = std::fwrite(buf.data(), 1, buf.size(), f);
    const int closed = std::fclose(f);
    if (w != buf.size() || closed != 0) return set_error(CS_ERR_INVALID, "write to %s failed", path);
    return CS_OK;
}
