// Frame and lineage files in the reference's text formats (utils.hpp:95-311 of both
// models), so that a run driven through abm_iterate writes the same files as the
// reference's runSimulation (simulation.hpp:1566-1573, 2025-2078):
//
//   cells      "# key = value" parameter lines, then one tab-separated row per cell:
//              the cell ID and group columns as integers, the columns between them as
//              doubles with 10 significant digits, further columns only when the
//              caller asks for them (as integers or doubles), rows ending in '\n'
//   lineage    one "child<TAB>parent" line per cell ID, in ID order
//
// Host code only (no device memory); the arrays are column-major like the rest of the C ABI.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/abm_capi.h"

namespace {

thread_local std::string g_err;

int io_fail(int code, const std::string& msg)
{
    g_err = msg;
    return code;
}

// ID and group columns of each model (indices.hpp: 3-D 0 and 20, 2-D 0 and 16)
bool layout(int dims, int& col_id, int& col_group)
{
    col_id = 0;
    if (dims == 3 || dims == 0) { col_group = 20; return true; }
    if (dims == 2) { col_group = 16; return true; }
    return false;
}

// std::ostream with setprecision(10) and the default float field prints a double as
// printf's "%.10g" does
void put_double(std::string& out, double v)
{
    char buf[40];
    std::snprintf(buf, sizeof(buf), "%.10g", v);
    out += buf;
}

void put_int(std::string& out, double v)
{
    char buf[24];
    std::snprintf(buf, sizeof(buf), "%d", static_cast<int>(v));
    out += buf;
}

}  // namespace

extern "C" const char* abm_io_last_error(void) { return g_err.c_str(); }

extern "C" int abm_write_cells(const char* path, const double* cells, int n, int ncols, int ld, int dims,
                               const char* params, const int* extra_cols, const int* extra_types, int n_extra)
{
    int col_id, col_group;
    if (!path || (n > 0 && !cells) || n < 0 || ld < n || n_extra < 0 || (n_extra > 0 && (!extra_cols || !extra_types)))
        return io_fail(ABM_ERR_ARG, "abm_write_cells: bad arguments");
    if (!layout(dims, col_id, col_group)) return io_fail(ABM_ERR_ARG, "abm_write_cells: dims must be 2 or 3");
    if (ncols <= col_group) return io_fail(ABM_ERR_ARG, "abm_write_cells: too few columns for the model");
    // which columns are written, and how: -1 skipped, 0 integer, 1 double
    std::vector<int> kind(ncols, -1);
    for (int j = 0; j < ncols; ++j)
        if (j == col_id || j == col_group) kind[j] = 0;
        else if (j > col_id && j < col_group) kind[j] = 1;
    for (int e = 0; e < n_extra; ++e)
    {
        const int j = extra_cols[e];
        if (j < 0 || j >= ncols) return io_fail(ABM_ERR_ARG, "abm_write_cells: extra column out of range");
        if (j == col_id || j == col_group || (j > col_id && j < col_group)) continue;   // written already
        kind[j] = extra_types[e] == 0 ? 0 : 1;
    }
    std::string out;
    // parameters: one "# key = value" line per line of `params` ("key = value" lines)
    if (params)
    {
        const char* p = params;
        while (*p)
        {
            const char* e = std::strchr(p, '\n');
            const size_t len = e ? (size_t)(e - p) : std::strlen(p);
            if (len > 0) { out += "# "; out.append(p, len); out += '\n'; }
            p += len + (e ? 1 : 0);
        }
    }
    for (int i = 0; i < n; ++i)
    {
        bool first = true;
        for (int j = 0; j < ncols; ++j)
        {
            if (kind[j] < 0) continue;
            if (!first) out += '\t';
            first = false;
            const double v = cells[(size_t)j * ld + i];
            if (kind[j] == 0) put_int(out, v);
            else put_double(out, v);
        }
        out += '\n';
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) return io_fail(ABM_ERR_ARG, std::string("abm_write_cells: cannot open ") + path + ": " + std::strerror(errno));
    const size_t w = std::fwrite(out.data(), 1, out.size(), f);
    const int c = std::fclose(f);
    if (w != out.size() || c != 0) return io_fail(ABM_ERR_ARG, std::string("abm_write_cells: write failed: ") + path);
    return ABM_OK;
}

extern "C" int abm_read_cells(const char* path, double* cells, int cap_rows, int cap_cols, int* n, int* ncols,
                              char* params, int params_cap)
{
    if (!path || !n || !ncols) return io_fail(ABM_ERR_ARG, "abm_read_cells: bad arguments");
    FILE* f = std::fopen(path, "rb");
    if (!f) return io_fail(ABM_ERR_ARG, std::string("abm_read_cells: cannot open ") + path + ": " + std::strerror(errno));
    std::string text;
    char buf[1 << 16];
    size_t r;
    while ((r = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, r);
    std::fclose(f);
    // utils.hpp:96-139: "# key = value" lines are parameters, the others tab-separated rows
    std::string ptext;
    int rows = 0, cols = 0;
    size_t pos = 0;
    while (pos < text.size())
    {
        size_t e = text.find('\n', pos);
        if (e == std::string::npos) e = text.size();
        std::string line = text.substr(pos, e - pos);
        pos = e + 1;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) continue;
        if (line[0] == '#')
        {
            const size_t eq = line.find(" = ");
            if (eq == std::string::npos || eq < 2) continue;
            ptext += line.substr(2, eq - 2) + " = " + line.substr(eq + 3) + "\n";
            continue;
        }
        // tokens split at tabs as std::getline(ss, token, '\t') splits them: a trailing tab
        // ends the row instead of starting an empty token; a blank line is skipped above,
        // where the reference would append a row of unset values
        int j = 0;
        size_t a = 0;
        while (a <= line.size())
        {
            if (a == line.size() && j > 0) break;
            size_t b = line.find('\t', a);
            if (b == std::string::npos) b = line.size();
            const std::string tok = line.substr(a, b - a);
            char* end = nullptr;
            const double v = std::strtod(tok.c_str(), &end);
            if (tok.empty() || end == tok.c_str())
                return io_fail(ABM_ERR_ARG, "abm_read_cells: not a number in row " + std::to_string(rows + 1));
            if (cells)
            {
                if (rows >= cap_rows || j >= cap_cols)
                    return io_fail(ABM_ERR_CAPACITY, "abm_read_cells: the file has more rows or columns than the buffer");
                cells[(size_t)j * cap_rows + rows] = v;
            }
            ++j;
            a = b + 1;
        }
        if (j > cols) cols = j;
        ++rows;
    }
    *n = rows;
    *ncols = cols;
    if (params)
    {
        if ((int)ptext.size() + 1 > params_cap)
            return io_fail(ABM_ERR_CAPACITY, "abm_read_cells: the parameter buffer is too small");
        std::memcpy(params, ptext.c_str(), ptext.size() + 1);
    }
    return ABM_OK;
}

extern "C" int abm_write_lineage(const char* path, const int* parents, int n)
{
    if (!path || n < 0 || (n > 0 && !parents)) return io_fail(ABM_ERR_ARG, "abm_write_lineage: bad arguments");
    std::string out;
    char buf[48];
    for (int i = 0; i < n; ++i)
    {
        std::snprintf(buf, sizeof(buf), "%d\t%d\n", i, parents[i]);   // utils.hpp:296-311
        out += buf;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) return io_fail(ABM_ERR_ARG, std::string("abm_write_lineage: cannot open ") + path + ": " + std::strerror(errno));
    const size_t w = std::fwrite(out.data(), 1, out.size(), f);
    const int c = std::fclose(f);
    if (w != out.size() || c != 0) return io_fail(ABM_ERR_ARG, std::string("abm_write_lineage: write failed: ") + path);
    return ABM_OK;
}

extern "C" int abm_read_lineage(const char* path, int* parents, int cap, int* n)
{
    if (!path || !n) return io_fail(ABM_ERR_ARG, "abm_read_lineage: bad arguments");
    FILE* f = std::fopen(path, "rb");
    if (!f) return io_fail(ABM_ERR_ARG, std::string("abm_read_lineage: cannot open ") + path + ": " + std::strerror(errno));
    // utils.hpp:265-288: "child<TAB>parent" per line; the result is indexed by child ID
    int child, parent, count = 0, max_child = -1;
    while (std::fscanf(f, "%d\t%d", &child, &parent) == 2)
    {
        if (child < 0) { std::fclose(f); return io_fail(ABM_ERR_ARG, "abm_read_lineage: negative cell ID"); }
        if (parents)
        {
            if (child >= cap)
            {
                std::fclose(f);
                return io_fail(ABM_ERR_CAPACITY, "abm_read_lineage: a cell ID exceeds the buffer");
            }
            parents[child] = parent;
        }
        if (child > max_child) max_child = child;
        ++count;
    }
    std::fclose(f);
    *n = max_child + 1;
    (void)count;
    return ABM_OK;
}
