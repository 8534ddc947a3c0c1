/*
 * Data import: pipe-separated text tables (the TPC-H / SSB .tbl format, one row per line,
 * fields separated by '|', a trailing '|' allowed) into device columns, through a binary
 * column cache.
 *
 * The reference's importer (db-engine-paradigms Import.cpp:165-250, parseColumns) reads
 * <dir>/<table>.tbl once, writes every column as a raw array to <dir>/cached/<table>_<column>
 * (runtime::Vector::writeBinary: the values, nothing else) and from then on maps those files;
 * each attribute's MinMaxInfo is the observed minimum and maximum (readBinary).  The same
 * layout is kept here, so a cache written by either side loads in the other, and the parse
 * runs on all host threads over byte ranges of the file split at line boundaries.
 *
 * Field types (schema "name:type,..." lists every field of a line in order; "-" skips one):
 *   int      32-bit integer                     -> VC_I32
 *   bigint   64-bit integer                     -> VC_I64
 *   date     YYYY-MM-DD as its Julian day number (the reference's types::Date) -> VC_I32
 *   decN     decimal with N fraction digits as an exact fixed-point integer (value * 10^N,
 *            the reference's types::Numeric<_, N>) -> VC_I64
 *   char     the field's first byte (types::Char<1>) -> VC_U8
 */
#include <algorithm>
#include <cerrno>
#include <cstring>
#include <fcntl.h>
#include <fstream>
#include <functional>
#include <sstream>
#include <sys/mman.h>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>

#include "engine_internal.hpp"
#include "../../include/voila_cuda.h"

struct vc_engine;

namespace vc {

int abi_guard_mlp(const std::function<void()>& f);
Engine& engine_of(vc_engine* e);
/* declares the table and its columns and uploads the data (engine.cpp) */
void import_declare(Engine& e, const std::string& table, int64_t rows, const std::vector<std::string>& names,
	const std::vector<int>& types, const std::vector<int64_t>& lo, const std::vector<int64_t>& hi,
	const std::vector<const void*>& data);

namespace {

struct FieldSpec {
	std::string name;
	enum Kind { Skip, Int, BigInt, Date, Dec, Char } kind = Skip;
	int scale = 0;
	int vtype() const { return kind == Char ? VC_TYPE_U8 : (kind == BigInt || kind == Dec) ? VC_TYPE_I64 : VC_TYPE_I32; }
	size_t width() const { return kind == Char ? 1 : (kind == BigInt || kind == Dec) ? 8 : 4; }
};

std::vector<FieldSpec> parse_schema(const std::string& s)
{
	std::vector<FieldSpec> out;
	std::stringstream ss(s);
	std::string item;
	while (std::getline(ss, item, ',')) {
		FieldSpec f;
		if (item == "-") {
			out.push_back(f);
			continue;
		}
		const size_t c = item.find(':');
		if (c == std::string::npos || c == 0) {
			throw Error(VC_ERR_INVALID, "import schema entries are name:type or -, got '" + item + "'");
		}
		f.name = item.substr(0, c);
		const std::string t = item.substr(c + 1);
		if (t == "int") {
			f.kind = FieldSpec::Int;
		} else if (t == "bigint") {
			f.kind = FieldSpec::BigInt;
		} else if (t == "date") {
			f.kind = FieldSpec::Date;
		} else if (t == "char") {
			f.kind = FieldSpec::Char;
		} else if (t.rfind("dec", 0) == 0 && t.size() > 3 && t.size() <= 5 &&
			t.find_first_not_of("0123456789", 3) == std::string::npos) {
			f.kind = FieldSpec::Dec;
			f.scale = std::stoi(t.substr(3));
			if (f.scale > 18) {
				throw Error(VC_ERR_INVALID, "decimal scale must be 0..18");
			}
		} else {
			throw Error(VC_ERR_INVALID, "unknown import type '" + t + "'");
		}
		out.push_back(f);
	}
	if (out.empty()) {
		throw Error(VC_ERR_INVALID, "empty import schema");
	}
	return out;
}

/* Julian day number of a Gregorian date (Fliegel and Van Flandern, CACM 11(10), 1968) */
int64_t julian_day(int64_t y, int64_t m, int64_t d)
{
	const int64_t a = (m - 14) / 12;
	return (1461 * (y + 4800 + a)) / 4 + (367 * (m - 2 - 12 * a)) / 12 - (3 * ((y + 4900 + a) / 100)) / 4 + d - 32075;
}

void trim(const char*& b, const char*& e)
{
	while (b < e && *b == ' ') b++;
	while (e > b && e[-1] == ' ') e--;
}

bool parse_int(const char* b, const char* e, int64_t& v)
{
	trim(b, e);
	bool neg = false;
	if (b < e && (*b == '-' || *b == '+')) {
		neg = *b == '-';
		b++;
	}
	if (b == e || e - b > 18) {
		return false;
	}
	int64_t x = 0;
	for (; b < e; b++) {
		if (*b < '0' || *b > '9') {
			return false;
		}
		x = x * 10 + (*b - '0');
	}
	v = neg ? -x : x;
	return true;
}

bool parse_dec(const char* b, const char* e, int scale, int64_t& v)
{
	trim(b, e);
	bool neg = false;
	if (b < e && (*b == '-' || *b == '+')) {
		neg = *b == '-';
		b++;
	}
	int64_t ip = 0, fp = 0;
	int fd = 0, id = 0;
	bool digits = false, dot = false;
	for (; b < e; b++) {
		if (*b == '.' && !dot) {
			dot = true;
		} else if (*b >= '0' && *b <= '9') {
			digits = true;
			if (!dot) {
				ip = ip * 10 + (*b - '0');
				if (++id + scale > 18) {
					return false;
				}
			} else if (fd < scale) {
				fp = fp * 10 + (*b - '0');
				fd++;
			} else if (*b != '0') {
				return false; /* more fraction digits than the scale holds exactly */
			}
		} else {
			return false;
		}
	}
	for (; fd < scale; fd++) {
		fp *= 10;
	}
	int64_t p10 = 1;
	for (int i = 0; i < scale; i++) {
		p10 *= 10;
	}
	v = ip * p10 + fp;
	if (neg) {
		v = -v;
	}
	return digits;
}

bool parse_date(const char* b, const char* e, int64_t& v)
{
	trim(b, e);
	int64_t part[3] = {0, 0, 0};
	int k = 0;
	bool any = false;
	for (; b < e; b++) {
		if (*b == '-') {
			if (++k > 2 || !any) {
				return false;
			}
			any = false;
		} else if (*b >= '0' && *b <= '9') {
			part[k] = part[k] * 10 + (*b - '0');
			any = true;
			if (part[k] > 99999) {
				return false;
			}
		} else {
			return false;
		}
	}
	if (k != 2 || !any || part[1] < 1 || part[1] > 12 || part[2] < 1 || part[2] > 31) {
		return false;
	}
	v = julian_day(part[0], part[1], part[2]);
	return true;
}

struct Chunk {
	std::vector<std::vector<unsigned char>> cols; /* per kept field: raw values */
	int64_t rows = 0;
	std::string error;
};

void parse_range(const char* b, const char* e, const std::vector<FieldSpec>& fs, size_t nkeep, Chunk& out,
	int64_t first_line)
{
	out.cols.assign(nkeep, {});
	int64_t line_no = first_line;
	while (b < e) {
		const char* nl = (const char*)std::memchr(b, '\n', (size_t)(e - b));
		const char* le = nl ? nl : e;
		if (le > b && le[-1] == '\r') {
			le--;
		}
		if (le > b) {
			const char* f = b;
			size_t ki = 0;
			for (size_t i = 0; i < fs.size(); i++) {
				const char* bar = (const char*)std::memchr(f, '|', (size_t)(le - f));
				const char* fe = bar ? bar : le;
				if (!bar && i + 1 < fs.size()) {
					out.error = "line " + std::to_string(line_no + 1) + " has fewer fields than the schema";
					return;
				}
				if (fs[i].kind != FieldSpec::Skip) {
					int64_t v = 0;
					bool ok = true;
					switch (fs[i].kind) {
					case FieldSpec::Int:
					case FieldSpec::BigInt: ok = parse_int(f, fe, v); break;
					case FieldSpec::Date: ok = parse_date(f, fe, v); break;
					case FieldSpec::Dec: ok = parse_dec(f, fe, fs[i].scale, v); break;
					case FieldSpec::Char: ok = fe > f; v = ok ? (unsigned char)*f : 0; break;
					default: break;
					}
					if (ok && fs[i].kind == FieldSpec::Int && (v < INT32_MIN || v > INT32_MAX)) {
						ok = false;
					}
					if (!ok) {
						out.error = "line " + std::to_string(line_no + 1) + ": cannot parse field " + fs[i].name;
						return;
					}
					auto& col = out.cols[ki++];
					const size_t w = fs[i].width();
					const size_t at = col.size();
					col.resize(at + w);
					if (w == 1) {
						col[at] = (unsigned char)v;
					} else if (w == 4) {
						const int32_t x = (int32_t)v;
						std::memcpy(&col[at], &x, 4);
					} else {
						std::memcpy(&col[at], &v, 8);
					}
				}
				f = bar ? bar + 1 : le;
			}
			out.rows++;
		}
		line_no++;
		b = nl ? nl + 1 : e;
	}
}

struct Mapped {
	void* p = nullptr;
	size_t n = 0;
	int fd = -1;
	~Mapped() {
		if (p && p != MAP_FAILED) {
			munmap(p, n);
		}
		if (fd >= 0) {
			close(fd);
		}
	}
};

bool map_file(const std::string& path, Mapped& m)
{
	m.fd = open(path.c_str(), O_RDONLY);
	if (m.fd < 0) {
		return false;
	}
	struct stat sb;
	if (fstat(m.fd, &sb) != 0) {
		return false;
	}
	m.n = (size_t)sb.st_size;
	if (m.n == 0) {
		return true;
	}
	m.p = mmap(nullptr, m.n, PROT_READ, MAP_PRIVATE, m.fd, 0);
	return m.p != MAP_FAILED;
}

void write_file(const std::string& path, const std::vector<unsigned char>& data)
{
	const std::string tmp = path + ".tmp" + std::to_string(getpid());
	{
		std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
		if (!f) {
			throw Error(VC_ERR_INVALID, "cannot write the column cache " + tmp);
		}
		f.write((const char*)data.data(), (std::streamsize)data.size());
	}
	if (std::rename(tmp.c_str(), path.c_str()) != 0) {
		throw Error(VC_ERR_INVALID, "cannot write the column cache " + path);
	}
}

} // namespace
} // namespace vc

extern "C" int vc_table_import(vc_engine* eng, const char* table, const char* dir, const char* schema, int threads,
	int64_t* rows_out)
{
	return vc::abi_guard_mlp([&] {
		using namespace vc;
		if (!eng || !table || !dir || !schema) {
			throw Error(VC_ERR_INVALID, "null argument");
		}
		const std::vector<FieldSpec> fs = parse_schema(schema);
		std::vector<int> keep;
		for (size_t i = 0; i < fs.size(); i++) {
			if (fs[i].kind != FieldSpec::Skip) {
				keep.push_back((int)i);
			}
		}
		if (keep.empty()) {
			throw Error(VC_ERR_INVALID, "the import schema keeps no field");
		}
		const std::string cache = std::string(dir) + "/cached/";
		std::vector<std::string> cpath;
		bool cached = true;
		for (int k : keep) {
			cpath.push_back(cache + table + "_" + fs[k].name);
			cached = cached && access(cpath.back().c_str(), R_OK) == 0;
		}
		std::vector<std::vector<unsigned char>> cols(keep.size());
		int64_t rows = -1;
		if (cached) {
			for (size_t i = 0; i < keep.size(); i++) {
				Mapped m;
				if (!map_file(cpath[i], m)) {
					throw Error(VC_ERR_INVALID, "cannot read the column cache " + cpath[i]);
				}
				const size_t w = fs[keep[i]].width();
				if (m.n % w) {
					throw Error(VC_ERR_INVALID, "column cache " + cpath[i] + " is not a whole number of values");
				}
				if (rows >= 0 && (int64_t)(m.n / w) != rows) {
					throw Error(VC_ERR_INVALID, std::string("the cached columns of ") + table + " differ in size");
				}
				rows = (int64_t)(m.n / w);
				if (m.n) {
					cols[i].assign((const unsigned char*)m.p, (const unsigned char*)m.p + m.n);
				}
			}
		} else {
			const std::string path = std::string(dir) + "/" + table + ".tbl";
			Mapped m;
			if (!map_file(path, m)) {
				throw Error(VC_ERR_INVALID, "cannot open " + path);
			}
			const char* base = (const char*)m.p;
			const size_t n = m.n;
			int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
			nt = (int)std::max<size_t>(1, std::min<size_t>((size_t)nt, n / (1 << 16) + 1));
			/* byte ranges split at line starts */
			std::vector<size_t> cut((size_t)nt + 1, 0);
			cut[(size_t)nt] = n;
			for (int t = 1; t < nt; t++) {
				size_t c = std::max(n * (size_t)t / (size_t)nt, cut[(size_t)t - 1]);
				while (c > 0 && c < n && base[c - 1] != '\n') {
					c++;
				}
				cut[(size_t)t] = c;
			}
			std::vector<Chunk> chunks((size_t)nt);
			std::vector<int64_t> first((size_t)nt, 0);
			for (int t = 1; t < nt; t++) { /* line numbers for error messages */
				first[(size_t)t] = first[(size_t)t - 1] + std::count(base + cut[(size_t)t - 1], base + cut[(size_t)t], '\n');
			}
			std::vector<std::thread> ws;
			for (int t = 0; t < nt; t++) {
				ws.emplace_back([&, t] {
					parse_range(base + cut[(size_t)t], base + cut[(size_t)t + 1], fs, keep.size(), chunks[(size_t)t],
						first[(size_t)t]);
				});
			}
			for (auto& w : ws) {
				w.join();
			}
			rows = 0;
			for (auto& c : chunks) {
				if (!c.error.empty()) {
					throw Error(VC_ERR_INVALID, std::string(table) + ".tbl " + c.error);
				}
				rows += c.rows;
			}
			for (size_t i = 0; i < keep.size(); i++) {
				for (auto& c : chunks) {
					cols[i].insert(cols[i].end(), c.cols[i].begin(), c.cols[i].end());
					std::vector<unsigned char>().swap(c.cols[i]);
				}
			}
			if (mkdir(cache.c_str(), 0777) != 0 && errno != EEXIST) {
				throw Error(VC_ERR_INVALID, "cannot create " + cache + ": " + std::strerror(errno));
			}
			for (size_t i = 0; i < keep.size(); i++) {
				write_file(cpath[i], cols[i]);
			}
		}
		/* declared domains: the observed minimum and maximum, as the reference's loader sets
		 * each attribute's MinMaxInfo */
		std::vector<std::string> names;
		std::vector<int> types;
		std::vector<int64_t> lo, hi;
		std::vector<const void*> data;
		for (size_t i = 0; i < keep.size(); i++) {
			const FieldSpec& f = fs[(size_t)keep[i]];
			int64_t mn = 0, mx = 0;
			for (int64_t r = 0; r < rows; r++) {
				int64_t v;
				if (f.width() == 1) {
					v = cols[i][(size_t)r];
				} else if (f.width() == 4) {
					int32_t x;
					std::memcpy(&x, &cols[i][(size_t)r * 4], 4);
					v = x;
				} else {
					std::memcpy(&v, &cols[i][(size_t)r * 8], 8);
				}
				if (r == 0 || v < mn) mn = v;
				if (r == 0 || v > mx) mx = v;
			}
			names.push_back(f.name);
			types.push_back(f.vtype());
			lo.push_back(mn);
			hi.push_back(mx);
			data.push_back(cols[i].data());
		}
		import_declare(engine_of(eng), table, rows, names, types, lo, hi, data);
		if (rows_out) {
			*rows_out = rows;
		}
	});
}
