/*
 * st_io.cu -- ParaView output of a cloud's parcels (the reference's write, A:1367-1430,
 * which uses WriteVTK.jl): one VTK XML UnstructuredGrid file per dump with a vertex cell per
 * parcel, point data "U" (velocity, 3 components) and "d" (diameter), and a .pvd collection
 * that lists the dumps by time.  Binary data are appended raw, little endian, with 64-bit
 * block headers, as WriteVTK writes them.  Host code over the public API.
 */
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <new>
#include <vector>

#include "scaletrack.h"

namespace st {
void st_set_last_error(const char* msg);
}

namespace {

int io_fail(const std::string& m)
{
    st::st_set_last_error(m.c_str());
    return ST_ERR_INVALID_ARGUMENT;
}

struct Block {
    const void* data;
    uint64_t bytes;
};

}  // namespace

extern "C" {

static int write_vtu_impl(st_handle* h, int cloud, const char* path);

int st_write_vtu(st_handle* h, int cloud, const char* path)
{
    try {
        return write_vtu_impl(h, cloud, path);
    } catch (const std::bad_alloc&) {
        st::st_set_last_error("st_write_vtu: out of host memory");
        return ST_ERR_OUT_OF_MEMORY;
    }
}

static int write_vtu_impl(st_handle* h, int cloud, const char* path)
{
    if (!h || !path) return io_fail("null argument to st_write_vtu");
    const int64_t n = st_num_parcels(h, cloud);
    if (n < 0) return io_fail("cloud out of range in st_write_vtu");
    std::vector<double> xyz(3 * n), uvw(3 * n), d(n);
    int rc = st_get_parcels(h, cloud, xyz.data(), uvw.data(), d.data());
    if (rc) return rc;
    /* interleave [3][n] into [n][3] as VTK wants */
    std::vector<double> pts(3 * n), vel(3 * n);
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            pts[3 * i + a] = xyz[a * n + i];
            vel[3 * i + a] = uvw[a * n + i];
        }
    std::vector<int64_t> conn(n), offs(n);
    std::vector<uint8_t> types(n, 1);   /* VTK_VERTEX */
    for (int64_t i = 0; i < n; ++i) {
        conn[i] = i;
        offs[i] = i + 1;
    }
    const Block blocks[] = {{pts.data(), (uint64_t)(24 * n)},   {conn.data(), (uint64_t)(8 * n)},
                            {offs.data(), (uint64_t)(8 * n)},   {types.data(), (uint64_t)n},
                            {vel.data(), (uint64_t)(24 * n)},   {d.data(), (uint64_t)(8 * n)}};
    uint64_t off[6];
    uint64_t pos = 0;
    for (int b = 0; b < 6; ++b) {
        off[b] = pos;
        pos += 8 + blocks[b].bytes;
    }
    FILE* f = fopen(path, "wb");
    if (!f) return io_fail(std::string("cannot open ") + path + " for writing");
    fprintf(f,
            "<?xml version=\"1.0\"?>\n"
            "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" "
            "header_type=\"UInt64\">\n"
            "  <UnstructuredGrid>\n"
            "    <Piece NumberOfPoints=\"%lld\" NumberOfCells=\"%lld\">\n"
            "      <Points>\n"
            "        <DataArray type=\"Float64\" Name=\"Points\" NumberOfComponents=\"3\" "
            "format=\"appended\" offset=\"%llu\"/>\n"
            "      </Points>\n"
            "      <Cells>\n"
            "        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"appended\" "
            "offset=\"%llu\"/>\n"
            "        <DataArray type=\"Int64\" Name=\"offsets\" format=\"appended\" "
            "offset=\"%llu\"/>\n"
            "        <DataArray type=\"UInt8\" Name=\"types\" format=\"appended\" "
            "offset=\"%llu\"/>\n"
            "      </Cells>\n"
            "      <PointData>\n"
            "        <DataArray type=\"Float64\" Name=\"U\" NumberOfComponents=\"3\" "
            "format=\"appended\" offset=\"%llu\"/>\n"
            "        <DataArray type=\"Float64\" Name=\"d\" format=\"appended\" "
            "offset=\"%llu\"/>\n"
            "      </PointData>\n"
            "    </Piece>\n"
            "  </UnstructuredGrid>\n"
            "  <AppendedData encoding=\"raw\">\n_",
            (long long)n, (long long)n, (unsigned long long)off[0], (unsigned long long)off[1],
            (unsigned long long)off[2], (unsigned long long)off[3], (unsigned long long)off[4],
            (unsigned long long)off[5]);
    bool ok = true;
    for (const Block& b : blocks) {
        ok = ok && fwrite(&b.bytes, 8, 1, f) == 1;
        if (b.bytes) ok = ok && fwrite(b.data, 1, b.bytes, f) == b.bytes;
    }
    fprintf(f, "\n  </AppendedData>\n</VTKFile>\n");
    ok = (fclose(f) == 0) && ok;
    if (!ok) return io_fail(std::string("short write to ") + path);
    return ST_OK;
}

int st_write_pvd(const char* path, int n, const double* times, const char* const* files)
{
    if (!path || n < 0 || (n > 0 && (!times || !files)))
        return io_fail("bad argument to st_write_pvd");
    FILE* f = fopen(path, "w");
    if (!f) return io_fail(std::string("cannot open ") + path + " for writing");
    fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"Collection\" version=\"1.0\" "
               "byte_order=\"LittleEndian\">\n  <Collection>\n");
    for (int i = 0; i < n; ++i)
        fprintf(f, "    <DataSet timestep=\"%.17g\" part=\"0\" file=\"%s\"/>\n", times[i],
                files[i] ? files[i] : "");
    fprintf(f, "  </Collection>\n</VTKFile>\n");
    if (fclose(f) != 0) return io_fail(std::string("short write to ") + path);
    return ST_OK;
}

}  // extern "C"
