// frame_io.cpp -- PyClaw's ascii frame files written by the library.
//
// Reference format: src/pyclaw/fileio/ascii.py:17-123 (write,
// write_patch_header, write_array): a patch header the caller supplies, then
// for each row j and each cell i of the row one line of the num_var values of
// (m, i, j) as "%18.8e", and a blank line after every row.  The reference
// formats value by value in Python; here the rows are formatted by several
// threads into private buffers and written in order, and a device patch's
// frame goes to the host and to the file while the solver keeps stepping
// (claw2_patch_write_ascii_async in claw2.cu).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <thread>
#include <vector>

#include "../../include/claw2.h"

extern "C" void claw2_internal_set_error(const char* msg);

namespace {

int io_fail(int code, const std::string& msg) {
    claw2_internal_set_error(msg.c_str());
    return code;
}

// rows [j0, j1) of a (nvar, mx, my) Fortran-ordered array
void format_rows(const double* q, int nvar, int mx, int j0, int j1, std::string& out) {
    char buf[64];
    out.clear();
    out.reserve((size_t)(j1 - j0) * ((size_t)mx * (18 * nvar + 1) + 1));
    for (int j = j0; j < j1; ++j) {
        for (int i = 0; i < mx; ++i) {
            const double* c = q + ((size_t)j * mx + i) * nvar;
            for (int m = 0; m < nvar; ++m) {
                const int n = std::snprintf(buf, sizeof buf, "%18.8e", c[m]);
                out.append(buf, (size_t)n);
            }
            out.push_back('\n');
        }
        out.push_back('\n');
    }
}

}  // namespace

// Shared with claw2.cu's asynchronous writer.
__attribute__((visibility("hidden"))) int claw2_internal_write_ascii(const char* path, int append,
                                                                     const char* header, const double* q,
                                                                     int nvar, int mx, int my, int nthreads) {
    if (!path || !header || !q || nvar < 1 || mx < 1 || my < 1)
        return io_fail(CLAW2_EINVAL, "bad arguments to the ascii writer");
    FILE* f = std::fopen(path, append ? "ab" : "wb");
    if (!f) return io_fail(CLAW2_EINVAL, std::string("cannot open ") + path + " for writing");
    bool ok = std::fputs(header, f) >= 0;
    unsigned hw = std::thread::hardware_concurrency();
    int nt = nthreads > 0 ? nthreads : (int)(hw ? hw : 1);
    nt = std::max(1, std::min(nt, my));
    // bounded chunks keep the buffers small: each pass formats nt blocks of rows
    const int rows_per_block = std::max(1, std::min(my, (int)(4u << 20) / std::max(1, mx * nvar * 18)));
    std::vector<std::string> bufs(nt);
    for (int j = 0; j < my && ok; j += nt * rows_per_block) {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) {
            const int j0 = std::min(my, j + t * rows_per_block), j1 = std::min(my, j0 + rows_per_block);
            if (j0 >= j1) {
                bufs[t].clear();
                continue;
            }
            if (nt == 1) format_rows(q, nvar, mx, j0, j1, bufs[t]);
            else th.emplace_back(format_rows, q, nvar, mx, j0, j1, std::ref(bufs[t]));
        }
        for (auto& x : th) x.join();
        for (int t = 0; t < nt && ok; ++t)
            ok = bufs[t].empty() || std::fwrite(bufs[t].data(), 1, bufs[t].size(), f) == bufs[t].size();
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return io_fail(CLAW2_EINVAL, std::string("write to ") + path + " failed");
    return CLAW2_OK;
}

extern "C" {

int claw2_write_ascii(const char* path, int append, const char* header, const double* q, int nvar, int mx,
                      int my, int nthreads) {
    return claw2_internal_write_ascii(path, append, header, q, nvar, mx, my, nthreads);
}

}  // extern "C"
