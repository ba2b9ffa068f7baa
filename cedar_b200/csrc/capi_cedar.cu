// capi_cedar.cu -- Cedar's C interface (include/cedar/capi.h) over the GPU
// solvers: integer handles for configs, topologies, vectors, matrices and
// solvers, with the reference's handle encoding (object kind in the top four
// bits, 1-based slot below; include/cedar/interface/object.h,
// src/interface/object.cc) and error codes.  Vectors and matrices are kept in
// host memory in Cedar's ghost-inclusive layout; cedar_solver_create sets up
// the GPU hierarchy from the matrix (cdr_gpu_solver_create_2d /
// cdr_gpu_solver3_create) with settings read from the config's JSON keys, and
// cedar_solver_run solves on the GPU from the vectors' host arrays.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cdr_gpu.h"
#include "../../include/cedar_capi.h"

namespace {

// ------------------------------------------------------------------ JSON
// A JSON value: enough of the format for Cedar's config files (objects,
// arrays, strings, numbers, true/false/null).
struct Json {
	enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
	bool b = false;
	double num = 0;
	std::string str;
	std::vector<Json> arr;
	std::map<std::string, Json> obj;
};

struct JsonParser {
	const std::string &s;
	size_t p = 0;
	bool ok = true;
	explicit JsonParser(const std::string &src) : s(src) {}
	void ws()
	{
		while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
	}
	bool lit(const char *w)
	{
		const size_t n = std::strlen(w);
		if (s.compare(p, n, w) != 0) return false;
		p += n;
		return true;
	}
	std::string string()
	{
		std::string out;
		++p;  // opening quote
		while (p < s.size() && s[p] != '"') {
			char c = s[p++];
			if (c == '\\' && p < s.size()) {
				const char e = s[p++];
				c = e == 'n' ? '\n' : e == 't' ? '\t' : e;
			}
			out.push_back(c);
		}
		if (p >= s.size()) ok = false;
		++p;
		return out;
	}
	Json value()
	{
		Json v;
		ws();
		if (p >= s.size()) { ok = false; return v; }
		const char c = s[p];
		if (c == '{') {
			v.kind = Json::OBJ;
			++p;
			ws();
			if (p < s.size() && s[p] == '}') { ++p; return v; }
			while (ok) {
				ws();
				if (p >= s.size() || s[p] != '"') { ok = false; break; }
				std::string k = string();
				ws();
				if (p >= s.size() || s[p] != ':') { ok = false; break; }
				++p;
				v.obj[k] = value();
				ws();
				if (p < s.size() && s[p] == ',') { ++p; continue; }
				if (p < s.size() && s[p] == '}') { ++p; break; }
				ok = false;
			}
		} else if (c == '[') {
			v.kind = Json::ARR;
			++p;
			ws();
			if (p < s.size() && s[p] == ']') { ++p; return v; }
			while (ok) {
				v.arr.push_back(value());
				ws();
				if (p < s.size() && s[p] == ',') { ++p; continue; }
				if (p < s.size() && s[p] == ']') { ++p; break; }
				ok = false;
			}
		} else if (c == '"') {
			v.kind = Json::STR;
			v.str = string();
		} else if (lit("true")) {
			v.kind = Json::BOOL;
			v.b = true;
		} else if (lit("false")) {
			v.kind = Json::BOOL;
		} else if (lit("null")) {
			v.kind = Json::NUL;
		} else {
			char *end = nullptr;
			v.num = std::strtod(s.c_str() + p, &end);
			if (end == s.c_str() + p) { ok = false; return v; }
			v.kind = Json::NUM;
			p = end - s.c_str();
		}
		return v;
	}
};

// value at a dotted path ("solver.cycle.nrelax-pre"), or nullptr
const Json *json_get(const Json &root, const std::string &path)
{
	const Json *n = &root;
	std::stringstream ss(path);
	std::string part;
	while (std::getline(ss, part, '.')) {
		if (n->kind != Json::OBJ) return nullptr;
		auto it = n->obj.find(part);
		if (it == n->obj.end()) return nullptr;
		n = &it->second;
	}
	return n;
}

// ---------------------------------------------------------------- objects
enum Kind { KIND_TOPO = 0x1, KIND_SOLVER = 0x2, KIND_MAT = 0x3, KIND_VEC = 0x4, KIND_CONFIG = 0x5 };
constexpr int KIND_SHIFT = 28;
constexpr unsigned KEY_MASK = 0x0fffffffu;

struct Object {
	virtual ~Object() {}
	int refcount = 0;
};

struct ConfigObj : Object {
	Json root;
};

struct TopoObj : Object {
	int nd = 2;
	unsigned n[3] = {0, 0, 1};  // interior points per dimension
	cedar_comm comm = 0;
	size_t len() const { return (size_t)(n[0] + 2) * (n[1] + 2) * (nd == 3 ? n[2] + 2 : 1); }
};

struct VecObj : Object {
	int nd = 2;
	cedar_topo topo = CEDAR_TOPO_NULL;
	unsigned n[3] = {0, 0, 1};
	std::vector<double> data;
};

struct MatObj : Object {
	int nd = 2;
	cedar_topo topo = CEDAR_TOPO_NULL;
	cedar_config conf = CEDAR_CONFIG_NULL;
	unsigned n[3] = {0, 0, 1};
	int nstencil = 5;
	std::vector<double> so;  // nstencil planes in Cedar's layout
	double *dso = nullptr;   // device copy for cedar_matvec, refreshed after a set
	bool dirty = true;
	~MatObj() override
	{
		if (dso) cudaFree(dso);
	}
	size_t plane() const { return (size_t)(n[0] + 2) * (n[1] + 2) * (nd == 3 ? n[2] + 2 : 1); }
};

struct SolverObj : Object {
	int nd = 2;
	cdr_gpu_solver *s2 = nullptr;
	cdr_gpu_solver3 *s3 = nullptr;
	unsigned n[3] = {0, 0, 1};
	int maxiter = 10;
	~SolverObj() override
	{
		if (s2) cdr_gpu_solver_destroy(s2);
		if (s3) cdr_gpu_solver3_destroy(s3);
	}
};

std::vector<std::unique_ptr<Object>> &objects()
{
	static std::vector<std::unique_ptr<Object>> o;
	return o;
}

int create(Kind k, Object *obj)
{
	objects().emplace_back(obj);
	return (int)(((unsigned)k << KIND_SHIFT) | (unsigned)objects().size());
}

template <typename T>
T *get(int handle, Kind k)
{
	if (((unsigned)handle >> KIND_SHIFT) != (unsigned)k) return nullptr;
	const size_t i = (unsigned)handle & KEY_MASK;
	if (i == 0 || i > objects().size()) return nullptr;
	return dynamic_cast<T *>(objects()[i - 1].get());
}

void incref(int handle)
{
	const size_t i = (unsigned)handle & KEY_MASK;
	if (i >= 1 && i <= objects().size() && objects()[i - 1]) objects()[i - 1]->refcount++;
}

void decref(int handle)
{
	const size_t i = (unsigned)handle & KEY_MASK;
	if (i >= 1 && i <= objects().size() && objects()[i - 1] && objects()[i - 1]->refcount > 0)
		objects()[i - 1]->refcount--;
}

// free the object of `handle` if nothing holds a reference to it
bool release(int handle)
{
	const size_t i = (unsigned)handle & KEY_MASK;
	if (i == 0 || i > objects().size() || !objects()[i - 1]) return false;
	if (objects()[i - 1]->refcount == 0) objects()[i - 1].reset();
	return true;
}

// -------------------------------------------------- settings from the config
// The keys and defaults of ml_settings::init (src/multilevel_settings.cc:15-61)
// and the GPU options ("gpu" object), as cedar_b200/config.py reads them.
int settings_from(const Json &c, int nd, cdr_gpu_settings *s)
{
	cdr_gpu_settings_default(s);
	auto str = [&](const char *path, const char *dflt) -> std::string {
		const Json *v = json_get(c, path);
		return v && v->kind == Json::STR ? v->str : std::string(dflt);
	};
	auto num = [&](const char *path, double dflt) -> double {
		const Json *v = json_get(c, path);
		return v && v->kind == Json::NUM ? v->num : dflt;
	};
	auto flag = [&](const char *path, bool dflt) -> bool {
		const Json *v = json_get(c, path);
		return v && v->kind == Json::BOOL ? v->b : dflt;
	};
	static const char *relax[] = {"point", "line-x", "line-y", "line-xy", "plane-xy", "plane-xz", "plane-yz",
	                              "plane-xyz"};
	const std::string r = str("solver.relaxation", "point");
	int ri = -1;
	for (int i = 0; i < 8; ++i)
		if (r == relax[i]) ri = i;
	if (ri < 0 || (nd == 2 && ri >= 4) || (nd == 3 && ri >= 1 && ri <= 3)) return CEDAR_ERR_CONFIG;
	s->relaxation = ri;
	const std::string cyc = str("solver.cycle.type", "v");
	if (cyc != "v" && cyc != "f") return CEDAR_ERR_CONFIG;
	s->cycle = cyc == "f" ? CDR_CYCLE_F : CDR_CYCLE_V;
	s->nrelax_pre = (int)num("solver.cycle.nrelax-pre", 2);
	s->nrelax_post = (int)num("solver.cycle.nrelax-post", 1);
	s->num_levels = (int)num("solver.num-levels", -1);
	s->maxiter = (int)num("solver.max-iter", 10);
	s->tol = num("solver.tol", 1e-8);
	s->min_coarse = (int)num("solver.min_coarse", 3);
	const std::string cg = str("solver.cg-solver", "LU");
	if (cg != "LU" && cg != "cedar" && cg != "redist") return CEDAR_ERR_CONFIG;
	const std::string prec = str("gpu.precision", "fp64");
	if (prec != "fp64" && prec != "fp32-ir") return CEDAR_ERR_CONFIG;
	s->precision = prec == "fp32-ir" ? CDR_PREC_F32_IR : CDR_PREC_F64;
	s->use_graph = flag("gpu.graph", true) ? 1 : 0;
	const std::string ls = str("gpu.line-solve", "scan");
	if (ls != "scan" && ls != "sequential") return CEDAR_ERR_CONFIG;
	s->line_flags = (ls == "sequential" ? CDR_LINES_EXACT : 0) | (flag("gpu.autotune", true) ? 0 : CDR_LINES_NOTUNE) |
	                (flag("gpu.line-stream", false) ? CDR_LINES_STREAM : 0);
	s->fuse_coarse = (int)num("gpu.fuse-coarse", 32);
	const std::string kr = str("gpu.krylov", "none");
	if (kr != "none" && kr != "fcg") return CEDAR_ERR_CONFIG;
	s->krylov = kr == "fcg" ? CDR_KRYLOV_FCG : CDR_KRYLOV_NONE;
	const std::string cs = str("gpu.coarse-solve", "banded");
	if (cs != "banded" && cs != "inverse") return CEDAR_ERR_CONFIG;
	s->coarse_solve = cs == "inverse" ? CDR_COARSE_INVERSE : CDR_COARSE_BANDED;
	s->fp32_levels = (int)num("gpu.fp32-levels", 0);
	s->krylov_replace = (int)num("gpu.fcg-replace", 1);
	const std::string fi = str("gpu.fine-iterate", "fp64");
	if (fi != "fp64" && fi != "fp32") return CEDAR_ERR_CONFIG;
	s->fp64_fine_iterate = fi == "fp64" ? 1 : 0;
	if (nd == 3 && (s->krylov != CDR_KRYLOV_NONE || s->coarse_solve != CDR_COARSE_BANDED || s->fp32_levels))
		return CEDAR_ERR_CONFIG;
	// kernel_params::periodic from grid.periodic (src/kernel_params.cc:72-74)
	if (const Json *pv = json_get(c, "grid.periodic")) {
		if (pv->kind != Json::ARR) return CEDAR_ERR_CONFIG;
		for (size_t i = 0; i < pv->arr.size() && i < 3; ++i)
			if (pv->arr[i].kind == Json::BOOL && pv->arr[i].b) s->periodic |= 1 << i;
		if (s->periodic >> nd) return CEDAR_ERR_CONFIG;
	}
	return CEDAR_SUCCESS;
}

}  // namespace

extern "C" {

int cedar_log_init(cedar_config conf) { return get<ConfigObj>(conf, KIND_CONFIG) ? CEDAR_SUCCESS : CEDAR_ERR_CONFIG; }

int cedar_config_create(const char *fname, cedar_config *newconfig)
{
	*newconfig = CEDAR_CONFIG_NULL;
	std::ifstream f(fname ? fname : "");
	if (!f.good()) return CEDAR_ERR_FNAME;
	std::stringstream ss;
	ss << f.rdbuf();
	const std::string text = ss.str();
	JsonParser jp(text);
	auto *c = new ConfigObj;
	c->root = jp.value();
	if (!jp.ok || c->root.kind != Json::OBJ) {
		delete c;
		return CEDAR_ERR_CONFIG;
	}
	*newconfig = create(KIND_CONFIG, c);
	return CEDAR_SUCCESS;
}

int cedar_config_get_int(cedar_config conf, const char *confpath, int *val)
{
	auto *c = get<ConfigObj>(conf, KIND_CONFIG);
	if (!c) return CEDAR_ERR_CONFIG;
	const Json *v = json_get(c->root, confpath ? confpath : "");
	if (!v || v->kind != Json::NUM) return CEDAR_ERR_CONFIG_PATH;
	*val = (int)v->num;
	return CEDAR_SUCCESS;
}

int cedar_config_free(cedar_config *conf)
{
	if (!get<ConfigObj>(*conf, KIND_CONFIG)) return CEDAR_ERR_CONFIG;
	release(*conf);
	*conf = CEDAR_CONFIG_NULL;
	return CEDAR_SUCCESS;
}

int cedar_topo_create2d(cedar_comm comm, unsigned int ngx, unsigned int ngy, unsigned int lnx[], unsigned int lny[],
                        int nprocx, int nprocy, cedar_topo *newtopo)
{
	*newtopo = CEDAR_TOPO_NULL;
	if (nprocx != 1 || nprocy != 1 || !lnx || !lny || lnx[0] != ngx || lny[0] != ngy || ngx < 1 || ngy < 1)
		return CEDAR_ERR_TOPO;
	auto *t = new TopoObj;
	t->nd = 2;
	t->n[0] = ngx;
	t->n[1] = ngy;
	t->comm = comm;
	*newtopo = create(KIND_TOPO, t);
	return CEDAR_SUCCESS;
}

int cedar_topo_create3d(cedar_comm comm, unsigned int ngx, unsigned int ngy, unsigned int ngz, unsigned int lnx[],
                        unsigned int lny[], unsigned int lnz[], int nprocx, int nprocy, int nprocz,
                        cedar_topo *newtopo)
{
	*newtopo = CEDAR_TOPO_NULL;
	if (nprocx != 1 || nprocy != 1 || nprocz != 1 || !lnx || !lny || !lnz || lnx[0] != ngx || lny[0] != ngy ||
	    lnz[0] != ngz || ngx < 1 || ngy < 1 || ngz < 1)
		return CEDAR_ERR_TOPO;
	auto *t = new TopoObj;
	t->nd = 3;
	t->n[0] = ngx;
	t->n[1] = ngy;
	t->n[2] = ngz;
	t->comm = comm;
	*newtopo = create(KIND_TOPO, t);
	return CEDAR_SUCCESS;
}

int cedar_topo_free(cedar_topo *topo)
{
	auto *t = get<TopoObj>(*topo, KIND_TOPO);
	if (!t) return CEDAR_ERR_TOPO;
	release(*topo);
	*topo = CEDAR_TOPO_NULL;
	return CEDAR_SUCCESS;
}

static int vec_create(cedar_topo topo, int nd, cedar_vec *vec)
{
	*vec = CEDAR_VEC_NULL;
	auto *t = get<TopoObj>(topo, KIND_TOPO);
	if (!t) return CEDAR_ERR_TOPO;
	if (t->nd != nd) return CEDAR_ERR_DIM;
	auto *v = new VecObj;
	v->nd = nd;
	v->topo = topo;
	std::memcpy(v->n, t->n, sizeof v->n);
	v->data.assign(t->len(), 0.0);
	incref(topo);
	*vec = create(KIND_VEC, v);
	return CEDAR_SUCCESS;
}

int cedar_vec_create2d(cedar_topo topo, cedar_vec *vec) { return vec_create(topo, 2, vec); }
int cedar_vec_create3d(cedar_topo topo, cedar_vec *vec) { return vec_create(topo, 3, vec); }

int cedar_vec_baseptr(cedar_vec vec, cedar_real **base)
{
	auto *v = get<VecObj>(vec, KIND_VEC);
	if (!v) return CEDAR_ERR_VEC;
	*base = v->data.data();
	return CEDAR_SUCCESS;
}

int cedar_vec_len2d(cedar_vec vec, cedar_len *ilen, cedar_len *jlen)
{
	auto *v = get<VecObj>(vec, KIND_VEC);
	if (!v) return CEDAR_ERR_VEC;
	if (v->nd != 2) return CEDAR_ERR_DIM;
	*ilen = v->n[0] + 2;
	*jlen = v->n[1] + 2;
	return CEDAR_SUCCESS;
}

int cedar_vec_len3d(cedar_vec vec, cedar_len *ilen, cedar_len *jlen, cedar_len *klen)
{
	auto *v = get<VecObj>(vec, KIND_VEC);
	if (!v) return CEDAR_ERR_VEC;
	if (v->nd != 3) return CEDAR_ERR_DIM;
	*ilen = v->n[0] + 2;
	*jlen = v->n[1] + 2;
	*klen = v->n[2] + 2;
	return CEDAR_SUCCESS;
}

int cedar_vec_getdim(cedar_vec vec, int *nd)
{
	auto *v = get<VecObj>(vec, KIND_VEC);
	if (!v) return CEDAR_ERR_VEC;
	*nd = v->nd;
	return CEDAR_SUCCESS;
}

int cedar_vec_free(cedar_vec *vec)
{
	auto *v = get<VecObj>(*vec, KIND_VEC);
	if (!v) return CEDAR_ERR_VEC;
	decref(v->topo);
	release(*vec);
	*vec = CEDAR_VEC_NULL;
	return CEDAR_SUCCESS;
}

static int mat_create(cedar_config conf, cedar_topo topo, int nd, int nstencil, cedar_mat *mat)
{
	*mat = CEDAR_MAT_NULL;
	auto *t = get<TopoObj>(topo, KIND_TOPO);
	if (!t) return CEDAR_ERR_TOPO;
	if (!get<ConfigObj>(conf, KIND_CONFIG)) return CEDAR_ERR_CONFIG;
	if (t->nd != nd) return CEDAR_ERR_DIM;
	auto *m = new MatObj;
	m->nd = nd;
	m->topo = topo;
	m->conf = conf;
	std::memcpy(m->n, t->n, sizeof m->n);
	m->nstencil = nstencil;
	m->so.assign(m->plane() * nstencil, 0.0);
	incref(topo);
	incref(conf);
	*mat = create(KIND_MAT, m);
	return CEDAR_SUCCESS;
}

int cedar_mat_create2d(cedar_config conf, cedar_topo topo, cedar_stencil_2d sten, cedar_mat *mat)
{
	if (sten != CEDAR_STENCIL_FIVE_PT && sten != CEDAR_STENCIL_NINE_PT) return CEDAR_ERR_STENCIL;
	return mat_create(conf, topo, 2, sten == CEDAR_STENCIL_FIVE_PT ? 3 : 5, mat);
}

int cedar_mat_create3d(cedar_config conf, cedar_topo topo, cedar_stencil_3d sten, cedar_mat *mat)
{
	if (sten != CEDAR_STENCIL_SEVEN_PT && sten != CEDAR_STENCIL_XXVII_PT) return CEDAR_ERR_STENCIL;
	return mat_create(conf, topo, 3, sten == CEDAR_STENCIL_SEVEN_PT ? 4 : 14, mat);
}

// Vertex-based entries into BoxMG's symmetric storage, as the reference's
// cedar_mat_set2d (src/2d/interface/c/mat.cc): off-diagonals negated; E, N,
// NE, SE and NW move to the neighbour's W, S, SW, NW and NW planes.
int cedar_mat_set2d(cedar_mat mat, unsigned int nvals, cedar_coord_2d coords[], cedar_real vals[])
{
	auto *m = get<MatObj>(mat, KIND_MAT);
	if (!m) return CEDAR_ERR_MAT;
	if (m->nd != 2) return CEDAR_ERR_DIM;
	const size_t ii = m->n[0] + 2, pl = m->plane();
	for (unsigned q = 0; q < nvals; ++q) {
		size_t ci = (size_t)coords[q].i + 1, cj = (size_t)coords[q].j + 1;
		if (coords[q].i >= m->n[0] || coords[q].j >= m->n[1]) return CEDAR_ERR_DIM;
		int dir = coords[q].dir;
		const double v = dir == BMG2_C ? vals[q] : -vals[q];
		switch (dir) {
		case BMG2_C: case BMG2_W: case BMG2_S: break;
		case BMG2_SW: if (m->nstencil == 3) return CEDAR_ERR_STENCIL; break;
		case BMG2_N: cj++; dir = BMG2_S; break;
		case BMG2_E: ci++; dir = BMG2_W; break;
		case BMG2_SE: if (m->nstencil == 3) return CEDAR_ERR_STENCIL; ci++; dir = BMG2_NW; break;
		case BMG2_NE: if (m->nstencil == 3) return CEDAR_ERR_STENCIL; ci++; cj++; dir = BMG2_SW; break;
		case BMG2_NW: if (m->nstencil == 3) return CEDAR_ERR_STENCIL; cj++; break;
		default: return CEDAR_ERR_STENCIL;
		}
		m->so[(size_t)dir * pl + cj * ii + ci] = v;
	}
	m->dirty = true;
	return CEDAR_SUCCESS;
}

// 3D: dir is the storage plane (src/3d/interface/c/mat.cc), off-diagonals negated
int cedar_mat_set3d(cedar_mat mat, unsigned int nvals, cedar_coord_3d coords[], cedar_real vals[])
{
	auto *m = get<MatObj>(mat, KIND_MAT);
	if (!m) return CEDAR_ERR_MAT;
	if (m->nd != 3) return CEDAR_ERR_DIM;
	const size_t ii = m->n[0] + 2, jj = m->n[1] + 2, pl = m->plane();
	for (unsigned q = 0; q < nvals; ++q) {
		if (coords[q].i >= m->n[0] || coords[q].j >= m->n[1] || coords[q].k >= m->n[2]) return CEDAR_ERR_DIM;
		const int dir = coords[q].dir;
		if (dir < 0 || dir >= m->nstencil) return CEDAR_ERR_STENCIL;
		const size_t ci = coords[q].i + 1, cj = coords[q].j + 1, ck = coords[q].k + 1;
		m->so[(size_t)dir * pl + (ck * jj + cj) * ii + ci] = dir == 0 ? vals[q] : -vals[q];
	}
	m->dirty = true;
	return CEDAR_SUCCESS;
}

int cedar_matvec(cedar_mat mat, cedar_vec x, cedar_vec y)
{
	auto *m = get<MatObj>(mat, KIND_MAT);
	if (!m) return CEDAR_ERR_MAT;
	auto *xv = get<VecObj>(x, KIND_VEC), *yv = get<VecObj>(y, KIND_VEC);
	if (!xv || !yv) return CEDAR_ERR_VEC;
	if (xv->nd != m->nd || yv->nd != m->nd || xv->data.size() != m->plane() || yv->data.size() != m->plane())
		return CEDAR_ERR_DIM;
	const size_t pl = m->plane(), bytes = pl * sizeof(double);
	if (!m->dso && cudaMalloc(&m->dso, bytes * m->nstencil) != cudaSuccess) return CEDAR_ERR_OTHER;
	if (m->dirty) {
		if (cudaMemcpy(m->dso, m->so.data(), bytes * m->nstencil, cudaMemcpyHostToDevice) != cudaSuccess)
			return CEDAR_ERR_OTHER;
		m->dirty = false;
	}
	// y = A x as -(0 - A x): the residual kernel with a zero right-hand side
	double *buf = nullptr;
	if (cudaMalloc(&buf, 3 * bytes) != cudaSuccess) return CEDAR_ERR_OTHER;
	double *dx = buf, *db = buf + pl, *dr = buf + 2 * pl;
	int rc = CEDAR_SUCCESS;
	if (cudaMemcpy(dx, xv->data.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemset(db, 0, 2 * bytes) != cudaSuccess)
		rc = CEDAR_ERR_OTHER;
	if (rc == CEDAR_SUCCESS) {
		const int r = m->nd == 2 ? cdr_gpu_residual_2d_f64(m->dso, m->nstencil, dx, db, dr, (int)m->n[0], (int)m->n[1],
		                                                    (int)m->n[0] + 2, nullptr, nullptr, 0)
		                         : cdr_gpu_residual_3d_f64(m->dso, m->nstencil, dx, db, dr, (int)m->n[0], (int)m->n[1],
		                                                    (int)m->n[2], (int)m->n[0] + 2, nullptr, nullptr, 0);
		if (r != CDR_OK || cudaMemcpy(yv->data.data(), dr, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
			rc = CEDAR_ERR_OTHER;
	}
	cudaFree(buf);
	if (rc != CEDAR_SUCCESS) return rc;
	for (double &v : yv->data) v = -v;  // interior: A x; ghost ring: 0
	return CEDAR_SUCCESS;
}

int cedar_mat_gettopo(cedar_mat mat, cedar_topo *topo)
{
	auto *m = get<MatObj>(mat, KIND_MAT);
	if (!m) {
		*topo = CEDAR_TOPO_NULL;
		return CEDAR_ERR_MAT;
	}
	*topo = m->topo;
	return CEDAR_SUCCESS;
}

// The operator as text, in the formats of the reference's dump: 2D rows of
// "index  i, j, " then the vertex-based stencil (src/2d/stencil_op.cc:5-50)
// into op-0-0.txt; 3D the stored planes, one value per line after the plane
// count and the value count (src/3d/util/io.cc:5-25) into so-0.0.0.
int cedar_mat_dump(cedar_mat mat)
{
	auto *m = get<MatObj>(mat, KIND_MAT);
	if (!m) return CEDAR_ERR_MAT;
	const size_t ii = m->n[0] + 2, pl = m->plane();
	if (m->nd == 2) {
		FILE *f = std::fopen("op-0-0.txt", "w");
		if (!f) return CEDAR_ERR_OTHER;
		auto S = [&](size_t i, size_t j, int d) { return m->so[(size_t)d * pl + j * ii + i]; };
		for (size_t j = 1; j <= m->n[1]; ++j)
			for (size_t i = 1; i <= m->n[0]; ++i) {
				std::fprintf(f, "%4zu %4zu, %4zu, ", (j - 1) * ii + i - 1, i + 1, j + 1);
				if (m->nstencil == 3)
					std::fprintf(f, "%.6e%.6e %.6e%.6e%.6e\n", -S(i, j + 1, BMG2_S), -S(i, j, BMG2_W), S(i, j, BMG2_C),
					             -S(i + 1, j, BMG2_W), -S(i, j, BMG2_S));
				else
					std::fprintf(f, "%.6e%.6e%.6e%.6e %.6e%.6e%.6e%.6e%.6e\n", -S(i, j + 1, BMG2_NW),
					             -S(i, j + 1, BMG2_S), -S(i + 1, j + 1, BMG2_SW), -S(i, j, BMG2_W), S(i, j, BMG2_C),
					             -S(i + 1, j, BMG2_W), -S(i, j, BMG2_SW), -S(i, j, BMG2_S), -S(i + 1, j, BMG2_NW));
			}
		std::fclose(f);
	} else {
		FILE *f = std::fopen("so-0.0.0", "w");
		if (!f) return CEDAR_ERR_OTHER;
		std::fprintf(f, "%d\n%zu\n", m->nstencil, m->so.size());
		for (double v : m->so) std::fprintf(f, "%.17g\n", v);
		std::fclose(f);
	}
	return CEDAR_SUCCESS;
}

int cedar_mat_free(cedar_mat *mat)
{
	auto *m = get<MatObj>(*mat, KIND_MAT);
	if (!m) return CEDAR_ERR_MAT;
	decref(m->topo);
	decref(m->conf);
	release(*mat);
	*mat = CEDAR_MAT_NULL;
	return CEDAR_SUCCESS;
}

int cedar_solver_create(cedar_mat mat, cedar_solver *solver)
{
	*solver = CEDAR_SOLVER_NULL;
	auto *m = get<MatObj>(mat, KIND_MAT);
	if (!m) return CEDAR_ERR_MAT;
	auto *c = get<ConfigObj>(m->conf, KIND_CONFIG);
	if (!c) return CEDAR_ERR_CONFIG;
	cdr_gpu_settings s;
	const int rc = settings_from(c->root, m->nd, &s);
	if (rc != CEDAR_SUCCESS) return rc;
	auto *so = new SolverObj;
	so->nd = m->nd;
	std::memcpy(so->n, m->n, sizeof so->n);
	so->maxiter = s.maxiter;
	const int r = m->nd == 2 ? cdr_gpu_solver_create_2d(&s, m->so.data(), m->nstencil, (int)m->n[0], (int)m->n[1], 0,
	                                                     &so->s2)
	                         : cdr_gpu_solver3_create(&s, m->so.data(), m->nstencil, (int)m->n[0], (int)m->n[1],
	                                                  (int)m->n[2], 0, &so->s3);
	if (r != CDR_OK) {
		delete so;
		return CEDAR_ERR_SOLVER;
	}
	*solver = create(KIND_SOLVER, so);
	return CEDAR_SUCCESS;
}

int cedar_solver_run(cedar_solver solver, cedar_vec x, cedar_vec b)
{
	auto *so = get<SolverObj>(solver, KIND_SOLVER);
	if (!so) return CEDAR_ERR_SOLVER;
	auto *xv = get<VecObj>(x, KIND_VEC), *bv = get<VecObj>(b, KIND_VEC);
	if (!xv || !bv) return CEDAR_ERR_VEC;
	if (xv->nd != so->nd || bv->nd != so->nd) return CEDAR_ERR_DIM;
	for (int d = 0; d < 3; ++d)
		if (xv->n[d] != so->n[d] || bv->n[d] != so->n[d]) return CEDAR_ERR_DIM;
	int iters = 0;
	const int r = so->nd == 2 ? cdr_gpu_solver_solve(so->s2, bv->data.data(), xv->data.data(), &iters, nullptr, 0)
	                          : cdr_gpu_solver3_solve(so->s3, bv->data.data(), xv->data.data(), &iters, nullptr, 0);
	return r == CDR_OK ? CEDAR_SUCCESS : CEDAR_ERR_SOLVER;
}

int cedar_solver_destroy(cedar_solver *solver)
{
	if (!get<SolverObj>(*solver, KIND_SOLVER)) return CEDAR_ERR_SOLVER;
	release(*solver);
	*solver = CEDAR_SOLVER_NULL;
	return CEDAR_SUCCESS;
}

int cedar_solver_free(cedar_solver *solver) { return cedar_solver_destroy(solver); }

}  // extern "C"
