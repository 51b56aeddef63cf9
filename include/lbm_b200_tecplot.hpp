// lbm_b200_tecplot.hpp -- the reference's Tecplot binary output ("#!TDV101",
// CPU/Inamuro.cpp:865-1013, Inamuro::writeTecplotBinary) for fields held in
// this library's layout, without the reference's CPU class.
//
// The file is the reference's byte for byte: version header, title "Inamuro",
// the variables X Y Z u v w rho fei press, one ordered zone "ZONE 001" of
// lx x ly x lz points in point packing, then per point (x fastest, then y,
// then z) the 1-based integer coordinates and u, v, w, rho, phi, p as float32.
// Strings are written as one 32-bit integer per character plus a 0
// terminator.  The byte order is the host's, as in the reference.
//
// Fields: lx*ly*lz doubles each, x fastest (cell = (z*ly + y)*lx + x, no ghost
// planes) -- the layout of lbm_download.  header-only; C++17.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace lbm_b200 {

namespace tecplot_detail {
inline void put_i32(std::vector<unsigned char>& b, int32_t v)
{
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    b.insert(b.end(), p, p + 4);
}
inline void put_f32(std::vector<unsigned char>& b, float v)
{
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    b.insert(b.end(), p, p + 4);
}
inline void put_text(std::vector<unsigned char>& b, const char* s)
{
    for (; *s; ++s) put_i32(b, static_cast<int32_t>(*s));
    put_i32(b, 0);
}
}  // namespace tecplot_detail

// The reference's output file name for a step: "3D" + 9-digit step + ".plt".
inline std::string tecplot_file_name(int step)
{
    char buf[32];
    std::snprintf(buf, sizeof(buf), "3D%09d.plt", step);
    return buf;
}

// Writes the Tecplot binary file of one state.  Returns false if the file
// cannot be written.
inline bool write_tecplot_binary(const std::string& path, int lx, int ly, int lz, const double* phi,
                                 const double* rho, const double* u, const double* v, const double* w,
                                 const double* p)
{
    using namespace tecplot_detail;
    std::vector<unsigned char> b;
    const size_t n = static_cast<size_t>(lx) * ly * lz;
    b.reserve(512 + n * 36);
    const char magic[] = "#!TDV101";
    b.insert(b.end(), magic, magic + 8);
    put_i32(b, 1);
    put_text(b, "Inamuro");
    const char* vars[] = {"X", "Y", "Z", "u", "v", "w", "rho", "fei", "press"};
    put_i32(b, 9);
    for (const char* s : vars) put_text(b, s);
    put_f32(b, 299.0f);   // zone marker
    put_text(b, "ZONE 001");
    const int32_t zone[] = {-1, 0, 1, 0, 0};   // colour, ordered zone, point packing, var location, face conn.
    for (int32_t v32 : zone) put_i32(b, v32);
    put_i32(b, lx);
    put_i32(b, ly);
    put_i32(b, lz);
    put_i32(b, 0);        // no auxiliary data
    put_f32(b, 357.0f);   // end of header
    put_f32(b, 299.0f);   // zone marker of the data section
    const int32_t formats[] = {3, 3, 3, 1, 1, 1, 1, 1, 1};   // X Y Z as integers, the rest float
    for (int32_t f : formats) put_i32(b, f);
    put_i32(b, 0);        // no variable sharing
    put_i32(b, -1);       // no connectivity sharing
    for (int z = 0; z < lz; ++z)
        for (int y = 0; y < ly; ++y)
            for (int x = 0; x < lx; ++x) {
                const size_t c = (static_cast<size_t>(z) * ly + y) * lx + x;
                put_i32(b, x + 1);
                put_i32(b, y + 1);
                put_i32(b, z + 1);
                const double vals[] = {u[c], v[c], w[c], rho[c], phi[c], p[c]};
                for (double d : vals) put_f32(b, static_cast<float>(d));
            }
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(b.data(), 1, b.size(), f) == b.size();
    return std::fclose(f) == 0 && ok;
}

}  // namespace lbm_b200
