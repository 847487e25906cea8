// io.cu -- mesh files: OFF (triangles / quads), TetGen (.node + .ele) and Medit (.mesh).
//
// Replaces the reference's parsers and writers (io/ParserOFF.cu:15-205, io/ParserTetGen.cu:13-120,
// io/ParserHex.cu:122-240, io/FileWriter.cu:12-147) and the file factories that use them
// (mesh/MeshFactory.cu:3-13,45-55,60-70,101-111). Host code only; the formats' conventions
// follow the reference:
//   * OFF: first line "OFF", then "nV nF nE", nV coordinate lines, nF faces "k v0 .. v(k-1)"
//     (k = 3 triangles, 4 quads; the first face decides, like getFaceType), 0-based;
//   * TetGen: <base>.node "nV 3 nAttr nMarker" then "i x y z [attr..] [marker]", <base>.ele
//     "nT 4 nAttr" then "i a b c d [attr..]"; indices are 1-based when the first node is
//     numbered 1 (startAtOne); attributes and boundary markers are read and not used (the
//     boundary is always derived from the boundary faces);
//   * Medit: keyword sections (MeshVersionFormatted, Dimension, Vertices, Triangles,
//     Quadrilaterals / Quads, Tetrahedra, Hexahedra, Edges, End), 1-based indices with a
//     reference number after each entry; hexahedra are stored with their two faces swapped
//     (file corners 4 5 6 7 0 1 2 3), as the reference's reader and writer do; the volume
//     section present wins over the surface ones.
// Writers print every float with 9 significant digits, so a written mesh reads back bit for bit
// (the reference's writers use the stream default of 6).
#include "capi_internal.cuh"
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

struct ParsedMesh {
    int elem_type = -1;
    std::vector<float> xyz;
    std::vector<int32_t> elems;
    int nV() const { return (int)(xyz.size() / 3); }
    int k() const { return elem_type == VSDMO_TRI ? 3 : elem_type == VSDMO_HEX ? 8 : 4; }
    int nE() const { return elem_type < 0 ? 0 : (int)(elems.size() / k()); }
};

struct IoError : std::runtime_error {
    explicit IoError(const std::string& m) : std::runtime_error(m) {}
};

bool read_file(const std::string& path, std::string& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

bool ends_with(const std::string& s, const std::string& t) {
    return s.size() >= t.size() && std::equal(t.rbegin(), t.rend(), s.rbegin(),
                                              [](char a, char b) { return std::tolower(a) == std::tolower(b); });
}

// Line reader over a buffer: '#' starts a comment, blank lines are skipped.
struct Lines {
    const std::string& s;
    size_t pos = 0;
    long line_no = 0;
    const std::string& name;
    Lines(const std::string& b, const std::string& n) : s(b), name(n) {}
    bool next(std::string& line) {
        while (pos < s.size()) {
            size_t e = s.find('\n', pos);
            if (e == std::string::npos) e = s.size();
            line.assign(s, pos, e - pos);
            pos = e + 1;
            ++line_no;
            const size_t h = line.find('#');
            if (h != std::string::npos) line.resize(h);
            size_t i = 0;
            while (i < line.size() && std::isspace((unsigned char)line[i])) ++i;
            if (i == line.size()) continue;
            line.erase(0, i);
            return true;
        }
        return false;
    }
    [[noreturn]] void fail(const std::string& what) const {
        throw IoError(name + ":" + std::to_string(line_no) + ": " + what);
    }
};

// numbers of one line
struct Tok {
    const char* p;
    const char* end;
    explicit Tok(const std::string& l) : p(l.c_str()), end(l.c_str() + l.size()) {}
    bool num_i(long& v) {
        char* e = nullptr;
        errno = 0;
        v = std::strtol(p, &e, 10);
        if (e == p || errno) return false;
        p = e;
        return true;
    }
    bool num_f(float& v) {
        char* e = nullptr;
        v = std::strtof(p, &e);
        if (e == p) return false;
        p = e;
        return true;
    }
};

int checked_count(long v, const Lines& L, const char* what) {
    if (v < 0 || v > INT32_MAX / 8) L.fail(std::string("bad ") + what + " count");
    return (int)v;
}

void parse_off(const std::string& path, ParsedMesh& m) {
    std::string buf, line;
    if (!read_file(path, buf)) throw IoError("cannot open " + path);
    Lines L(buf, path);
    if (!L.next(line) || line.compare(0, 3, "OFF") != 0) L.fail("first line is not OFF");
    if (!L.next(line)) L.fail("missing counts");
    long nv, nf, ne;
    {
        Tok t(line);
        if (!t.num_i(nv) || !t.num_i(nf) || !t.num_i(ne)) L.fail("expected nVertices nFaces nEdges");
    }
    const int nV = checked_count(nv, L, "vertex"), nF = checked_count(nf, L, "face");
    m.xyz.resize(3 * (size_t)nV);
    for (int i = 0; i < nV; ++i) {
        if (!L.next(line)) L.fail("missing vertex lines");
        Tok t(line);
        if (!t.num_f(m.xyz[3 * (size_t)i]) || !t.num_f(m.xyz[3 * (size_t)i + 1]) || !t.num_f(m.xyz[3 * (size_t)i + 2]))
            L.fail("expected x y z");
    }
    int k = 0;
    for (int f = 0; f < nF; ++f) {
        if (!L.next(line)) L.fail("missing face lines");
        Tok t(line);
        long kk;
        if (!t.num_i(kk)) L.fail("expected a face");
        if (f == 0) {
            if (kk != 3 && kk != 4) L.fail("faces must be triangles or quads");
            k = (int)kk;
            m.elem_type = k == 3 ? VSDMO_TRI : VSDMO_QUAD;
            m.elems.resize((size_t)nF * k);
        } else if (kk != k) {
            L.fail("faces of mixed size");
        }
        for (int a = 0; a < k; ++a) {
            long v;
            if (!t.num_i(v)) L.fail("expected a vertex index");
            if (v < 0 || v >= nV) L.fail("vertex index out of range");
            m.elems[(size_t)f * k + a] = (int32_t)v;
        }
    }
    if (nF == 0) L.fail("no faces");
}

std::string tetgen_base(const std::string& path) {
    if (ends_with(path, ".node") || ends_with(path, ".ele")) return path.substr(0, path.find_last_of('.'));
    return path;
}

void parse_tetgen(const std::string& path, ParsedMesh& m) {
    const std::string base = tetgen_base(path);
    std::string nbuf, ebuf, line;
    if (!read_file(base + ".node", nbuf)) throw IoError("cannot open " + base + ".node");
    if (!read_file(base + ".ele", ebuf)) throw IoError("cannot open " + base + ".ele");
    bool one_based = false;
    int nV = 0;
    {
        Lines L(nbuf, base + ".node");
        if (!L.next(line)) L.fail("missing header");
        long n, dim, nattr, nmark = 0;
        Tok t(line);
        if (!t.num_i(n) || !t.num_i(dim) || !t.num_i(nattr)) L.fail("expected nPoints dim nAttributes [nMarkers]");
        t.num_i(nmark);
        if (dim != 3) L.fail("dimension must be 3");
        nV = checked_count(n, L, "point");
        m.xyz.resize(3 * (size_t)nV);
        for (int i = 0; i < nV; ++i) {
            if (!L.next(line)) L.fail("missing point lines");
            Tok p(line);
            long id;
            if (!p.num_i(id)) L.fail("expected a point number");
            if (i == 0) one_based = id == 1;
            if (!p.num_f(m.xyz[3 * (size_t)i]) || !p.num_f(m.xyz[3 * (size_t)i + 1]) || !p.num_f(m.xyz[3 * (size_t)i + 2]))
                L.fail("expected x y z");
        }
    }
    {
        Lines L(ebuf, base + ".ele");
        if (!L.next(line)) L.fail("missing header");
        long n, per;
        Tok t(line);
        if (!t.num_i(n) || !t.num_i(per)) L.fail("expected nTetrahedra nodesPerTet");
        if (per != 4) L.fail("only 4-node tetrahedra are supported");
        const int nT = checked_count(n, L, "tetrahedron");
        if (nT == 0) L.fail("no tetrahedra");
        m.elem_type = VSDMO_TET;
        m.elems.resize(4 * (size_t)nT);
        for (int e = 0; e < nT; ++e) {
            if (!L.next(line)) L.fail("missing tetrahedron lines");
            Tok p(line);
            long id;
            if (!p.num_i(id)) L.fail("expected a tetrahedron number");
            for (int a = 0; a < 4; ++a) {
                long v;
                if (!p.num_i(v)) L.fail("expected a node index");
                if (one_based) --v;
                if (v < 0 || v >= nV) L.fail("node index out of range");
                m.elems[4 * (size_t)e + a] = (int32_t)v;
            }
        }
    }
}

// whitespace-separated tokens with '#' comments (Medit is keyword / count / values)
struct Words {
    const std::string& s;
    size_t pos = 0;
    const std::string& name;
    Words(const std::string& b, const std::string& n) : s(b), name(n) {}
    bool next(std::string& w) {
        for (;;) {
            while (pos < s.size() && std::isspace((unsigned char)s[pos])) ++pos;
            if (pos >= s.size()) return false;
            if (s[pos] == '#') {
                while (pos < s.size() && s[pos] != '\n') ++pos;
                continue;
            }
            const size_t b = pos;
            while (pos < s.size() && !std::isspace((unsigned char)s[pos])) ++pos;
            w.assign(s, b, pos - b);
            return true;
        }
    }
    long integer() {
        std::string w;
        if (!next(w)) throw IoError(name + ": unexpected end of file");
        char* e = nullptr;
        const long v = std::strtol(w.c_str(), &e, 10);
        if (*e) throw IoError(name + ": expected an integer, found '" + w + "'");
        return v;
    }
    float real() {
        std::string w;
        if (!next(w)) throw IoError(name + ": unexpected end of file");
        char* e = nullptr;
        const float v = std::strtof(w.c_str(), &e);
        if (*e) throw IoError(name + ": expected a number, found '" + w + "'");
        return v;
    }
};

void parse_medit(const std::string& path, ParsedMesh& m) {
    std::string buf, w;
    if (!read_file(path, buf)) throw IoError("cannot open " + path);
    Words W(buf, path);
    int dim = 3, nV = -1;
    std::vector<int32_t> sec[4];   // triangles, quads, tets, hexes
    auto count = [&](const char* what) {
        const long n = W.integer();
        if (n < 0 || n > INT32_MAX / 8) throw IoError(path + ": bad " + what + " count");
        return (int)n;
    };
    auto read_elems = [&](int k, std::vector<int32_t>& out, bool swap_faces) {
        const int n = count("element");
        out.resize((size_t)n * k);
        for (int e = 0; e < n; ++e) {
            int32_t v[8];
            for (int a = 0; a < k; ++a) v[a] = (int32_t)(W.integer() - 1);
            (void)W.integer();   // reference number
            for (int a = 0; a < k; ++a) out[(size_t)e * k + a] = swap_faces ? v[(a + 4) % 8] : v[a];
        }
    };
    while (W.next(w)) {
        if (w == "MeshVersionFormatted") (void)W.integer();
        else if (w == "Dimension") {
            dim = (int)W.integer();
            if (dim != 2 && dim != 3) throw IoError(path + ": dimension must be 2 or 3");
        } else if (w == "Vertices") {
            nV = count("vertex");
            m.xyz.assign(3 * (size_t)nV, 0.f);
            for (int i = 0; i < nV; ++i) {
                for (int a = 0; a < dim; ++a) m.xyz[3 * (size_t)i + a] = W.real();
                (void)W.integer();
            }
        } else if (w == "Edges") {
            const int n = count("edge");
            for (int e = 0; e < n; ++e) { W.integer(); W.integer(); W.integer(); }
        } else if (w == "Triangles") read_elems(3, sec[0], false);
        else if (w == "Quadrilaterals" || w == "Quads") read_elems(4, sec[1], false);
        else if (w == "Tetrahedra") read_elems(4, sec[2], false);
        else if (w == "Hexahedra") read_elems(8, sec[3], true);
        else if (w == "End") break;
        else throw IoError(path + ": unsupported section '" + w + "'");
    }
    if (nV < 0) throw IoError(path + ": no Vertices section");
    const int order[4] = { 3, 2, 1, 0 };
    const int types[4] = { VSDMO_TRI, VSDMO_QUAD, VSDMO_TET, VSDMO_HEX };
    for (int s : order)
        if (!sec[s].empty()) {
            m.elem_type = types[s];
            m.elems = std::move(sec[s]);
            break;
        }
    if (m.elem_type < 0) throw IoError(path + ": no element section");
    std::vector<char> used(nV, 0);
    for (int32_t v : m.elems) {
        if (v < 0 || v >= nV) throw IoError(path + ": element index out of range");
        used[v] = 1;
    }
    // the reference's hex reader rejects unreferenced vertices (io/ParserHex.cu:216-230)
    if (m.elem_type == VSDMO_HEX)
        for (char u : used)
            if (!u) throw IoError(path + ": the file has vertices that no hexahedron uses");
}

int detect_format(const std::string& path, int format) {
    if (format != VSDMO_FMT_AUTO) return format;
    if (ends_with(path, ".off")) return VSDMO_FMT_OFF;
    if (ends_with(path, ".mesh")) return VSDMO_FMT_MEDIT;
    if (ends_with(path, ".node") || ends_with(path, ".ele")) return VSDMO_FMT_TETGEN;
    std::ifstream f(path + ".node");
    if (f.is_open()) return VSDMO_FMT_TETGEN;
    return -1;
}

void parse_any(const std::string& path, int format, ParsedMesh& m) {
    switch (detect_format(path, format)) {
    case VSDMO_FMT_OFF: parse_off(path, m); break;
    case VSDMO_FMT_TETGEN: parse_tetgen(path, m); break;
    case VSDMO_FMT_MEDIT: parse_medit(path, m); break;
    default: throw IoError("cannot tell the format of " + path + " (.off, .mesh, .node/.ele)");
    }
}

void write_any(const std::string& path, int format, int type, const float* xyz, int nV, const int32_t* el, int nE) {
    const int k = type == VSDMO_TRI ? 3 : type == VSDMO_HEX ? 8 : 4;
    format = detect_format(path, format);
    if (format < 0) {
        format = type == VSDMO_TET ? VSDMO_FMT_TETGEN : type == VSDMO_HEX ? VSDMO_FMT_MEDIT : VSDMO_FMT_OFF;
    }
    auto open = [](const std::string& p) {
        FILE* f = std::fopen(p.c_str(), "w");
        if (!f) throw IoError("cannot write " + p);
        return f;
    };
    auto close = [](FILE* f, const std::string& p) {
        if (std::ferror(f) | std::fclose(f)) throw IoError("error writing " + p);
    };
    if (format == VSDMO_FMT_OFF) {
        if (type != VSDMO_TRI && type != VSDMO_QUAD) throw IoError("OFF holds triangle or quad meshes");
        FILE* f = open(path);
        std::fprintf(f, "OFF\n%d %d 0\n", nV, nE);
        for (int i = 0; i < nV; ++i) std::fprintf(f, "%.9g %.9g %.9g\n", xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2]);
        for (int e = 0; e < nE; ++e) {
            std::fprintf(f, "%d", k);
            for (int a = 0; a < k; ++a) std::fprintf(f, " %d", el[(size_t)e * k + a]);
            std::fputc('\n', f);
        }
        close(f, path);
    } else if (format == VSDMO_FMT_TETGEN) {
        if (type != VSDMO_TET) throw IoError("TetGen files hold tetrahedral meshes");
        const std::string base = tetgen_base(path);
        FILE* f = open(base + ".node");
        std::fprintf(f, "# written by libvsdmo\n%d 3 0 0\n", nV);
        for (int i = 0; i < nV; ++i)
            std::fprintf(f, "%d %.9g %.9g %.9g\n", i, xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2]);
        close(f, base + ".node");
        f = open(base + ".ele");
        std::fprintf(f, "# written by libvsdmo\n%d 4 0\n", nE);
        for (int e = 0; e < nE; ++e)
            std::fprintf(f, "%d %d %d %d %d\n", e, el[4 * (size_t)e], el[4 * (size_t)e + 1], el[4 * (size_t)e + 2], el[4 * (size_t)e + 3]);
        close(f, base + ".ele");
    } else {
        FILE* f = open(path);
        std::fprintf(f, "MeshVersionFormatted 1\nDimension 3\nVertices %d\n", nV);
        for (int i = 0; i < nV; ++i)
            std::fprintf(f, "%.9g %.9g %.9g 0\n", xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2]);
        const char* names[4] = { "Triangles", "Quadrilaterals", "Tetrahedra", "Hexahedra" };
        std::fprintf(f, "%s %d\n", names[type], nE);
        for (int e = 0; e < nE; ++e) {
            for (int a = 0; a < k; ++a) {
                const int src = type == VSDMO_HEX ? (a + 4) % 8 : a;
                std::fprintf(f, "%d ", el[(size_t)e * k + src] + 1);
            }
            std::fprintf(f, "0\n");
        }
        std::fprintf(f, "End\n");
        close(f, path);
    }
}

template <class F>
vsdmo_status io_guarded(F&& f) {
    try {
        f();
        g_last_error.clear();
        return VSDMO_OK;
    } catch (const IoError& e) {
        return fail(VSDMO_E_IO, e.what());
    } catch (const Error& e) {
        return fail(e.status, e.what());
    } catch (const std::bad_alloc&) {
        return fail(VSDMO_E_NOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(VSDMO_E_IO, e.what());
    }
}

__global__ void k_surface_positions(const float4* pos, int n, float* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pos[i];
        out[3 * i] = p.x; out[3 * i + 1] = p.y; out[3 * i + 2] = p.z;
    }
}

}  // namespace

VSDMO_API vsdmo_status vsdmo_file_read(const char* path, int format, int* elem_type, int* n_vertices, int* n_elements,
                                       float* xyz, int32_t* elems) {
    if (!path || !elem_type || !n_vertices || !n_elements) return fail(VSDMO_E_ARG, "null argument");
    if (format < VSDMO_FMT_AUTO || format > VSDMO_FMT_MEDIT) return fail(VSDMO_E_ARG, "bad format");
    return io_guarded([&] {
        ParsedMesh m;
        parse_any(path, format, m);
        *elem_type = m.elem_type;
        *n_vertices = m.nV();
        *n_elements = m.nE();
        if (xyz) std::memcpy(xyz, m.xyz.data(), sizeof(float) * m.xyz.size());
        if (elems) std::memcpy(elems, m.elems.data(), sizeof(int32_t) * m.elems.size());
    });
}

VSDMO_API vsdmo_status vsdmo_file_write(const char* path, int format, int elem_type, const float* xyz, int n_vertices,
                                        const int32_t* elems, int n_elements) {
    if (!path || !xyz || !elems || n_vertices <= 0 || n_elements <= 0) return fail(VSDMO_E_ARG, "null or empty argument");
    if (format < VSDMO_FMT_AUTO || format > VSDMO_FMT_MEDIT) return fail(VSDMO_E_ARG, "bad format");
    if (elem_type < VSDMO_TRI || elem_type > VSDMO_HEX) return fail(VSDMO_E_ARG, "bad element type");
    return io_guarded([&] { write_any(path, format, elem_type, xyz, n_vertices, elems, n_elements); });
}

VSDMO_API vsdmo_status vsdmo_mesh_create_from_file(const char* path, int format, uint32_t color_seed, void* cuda_stream,
                                                   vsdmo_mesh_t* out) {
    if (!out) return fail(VSDMO_E_ARG, "null output handle");
    *out = nullptr;
    if (!path) return fail(VSDMO_E_ARG, "null path");
    if (format < VSDMO_FMT_AUTO || format > VSDMO_FMT_MEDIT) return fail(VSDMO_E_ARG, "bad format");
    ParsedMesh m;
    const vsdmo_status st = io_guarded([&] { parse_any(path, format, m); });
    if (st != VSDMO_OK) return st;
    return vsdmo_mesh_create(m.elem_type, m.xyz.data(), m.nV(), m.elems.data(), m.nE(), VSDMO_HOST, color_seed,
                             cuda_stream, out);
}

VSDMO_API vsdmo_status vsdmo_mesh_write_file(vsdmo_mesh_t mesh, const char* path, int format) {
    if (!mesh || !path) return fail(VSDMO_E_ARG, "null argument");
    if (format < VSDMO_FMT_AUTO || format > VSDMO_FMT_MEDIT) return fail(VSDMO_E_ARG, "bad format");
    return io_guarded([&] {
        const Mesh& m = mesh->m;
        // positions and elements in the caller's numbering
        std::vector<float> xyz(3 * (size_t)m.nV);
        std::vector<float> pos = [&] {
            std::vector<float4> p = m.pos.to_host();
            std::vector<float> o(3 * p.size());
            for (size_t i = 0; i < p.size(); ++i) { o[3 * i] = p[i].x; o[3 * i + 1] = p[i].y; o[3 * i + 2] = p[i].z; }
            return o;
        }();
        const std::vector<int> new_of_old = m.new_of_old.to_host();
        std::vector<int> old_of_new(m.nV);
        for (int i = 0; i < m.nV; ++i) {
            old_of_new[new_of_old[i]] = i;
            std::memcpy(&xyz[3 * (size_t)i], &pos[3 * (size_t)new_of_old[i]], 3 * sizeof(float));
        }
        std::vector<int32_t> el = m.elems.to_host();
        for (auto& v : el) v = old_of_new[v];
        write_any(path, format, m.type, xyz.data(), m.nV, el.data(), m.nE);
    });
}

VSDMO_API vsdmo_status vsdmo_mesh_create_surface(vsdmo_mesh_t volume, uint32_t color_seed, void* cuda_stream,
                                                 vsdmo_mesh_t* out) {
    if (!out) return fail(VSDMO_E_ARG, "null output handle");
    *out = nullptr;
    if (!volume) return fail(VSDMO_E_ARG, "null mesh");
    const Mesh& m = volume->m;
    if (m.type != VSDMO_TET && m.type != VSDMO_HEX) return fail(VSDMO_E_ARG, "the mesh has no volume elements");
    std::vector<float> xyz;
    std::vector<int> faces;
    const vsdmo_status st = guarded([&] {
        DBuf<float> d(3L * std::max(m.nSurf, 1), m.stream);
        k_surface_positions<<<grid_for(m.nSurf, 256), 256, 0, m.stream>>>(m.pos.p, m.nSurf, d.p);
        VSDMO_CHECK_LAUNCH();
        xyz = d.to_host();
        faces = m.tris.to_host();
    });
    if (st != VSDMO_OK) return st;
    return vsdmo_mesh_create(m.fk == 3 ? VSDMO_TRI : VSDMO_QUAD, xyz.data(), m.nSurf, faces.data(),
                             (int)(faces.size() / m.fk), VSDMO_HOST, color_seed, cuda_stream, out);
}
