/*
 * Run-time compilation of generated pipeline kernels with NVRTC for sm_100a.
 *
 * The CUDA flavor's counterpart of Compiler::call_cxx_compiler + dlopen
 * (compiler.cpp:19-57, :291-311): generated source is compiled to a cubin, loaded as a
 * CUDA library and its kernels looked up by name.  Compiled cubins are cached in memory
 * and on disk (VOILA_B200_JIT_CACHE, default ~/.cache/voila_b200_jit) keyed by a hash of
 * the source and the compile options, so a plan shape compiles once.
 */
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <sys/stat.h>
#include <unistd.h>

#include <nvrtc.h>

#include "engine_internal.hpp"

namespace vc {

#include "device_header.inc" /* kDeviceHeader: voila_device.cuh as a string */

const std::string& device_header_source()
{
	static const std::string s(kDeviceHeader);
	return s;
}

static uint64_t fnv1a(const std::string& s, uint64_t h = 1469598103934665603ull)
{
	for (unsigned char c : s) {
		h ^= c;
		h *= 1099511628211ull;
	}
	return h;
}

static const char* kOpts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "--device-int128",
	"-DVOILA_B200_NVRTC=1"};
static const int kNumOpts = 5;

static std::string cache_dir()
{
	const char* env = std::getenv("VOILA_B200_JIT_CACHE");
	if (env && *env) {
		return env;
	}
	const char* home = std::getenv("HOME");
	return std::string(home && *home ? home : "/tmp") + "/.cache/voila_b200_jit";
}

static void mkdirs(const std::string& path)
{
	std::string cur;
	std::stringstream ss(path);
	std::string part;
	if (!path.empty() && path[0] == '/') {
		cur = "/";
	}
	while (std::getline(ss, part, '/')) {
		if (part.empty()) {
			continue;
		}
		cur += part + "/";
		mkdir(cur.c_str(), 0755);
	}
}

static std::string key_of(const std::string& source)
{
	int major = 0, minor = 0;
	nvrtcVersion(&major, &minor);
	std::string opts;
	for (int i = 0; i < kNumOpts; i++) {
		opts += kOpts[i];
		opts += ' ';
	}
	uint64_t h = fnv1a(source);
	h = fnv1a(device_header_source(), h);
	h = fnv1a(opts + std::to_string(major) + "." + std::to_string(minor), h);
	char buf[32];
	std::snprintf(buf, sizeof(buf), "%016llx", (unsigned long long)h);
	return buf;
}

std::string jit_cubin(const std::string& source, std::string* log_out)
{
	const std::string key = key_of(source);
	const std::string dir = cache_dir();
	const std::string path = dir + "/" + key + ".cubin";
	{
		std::ifstream in(path, std::ios::binary);
		if (in) {
			std::stringstream ss;
			ss << in.rdbuf();
			std::string bin = ss.str();
			if (bin.size() > 16) {
				return bin;
			}
		}
	}
	nvrtcProgram prog;
	const char* hdr_src[] = {kDeviceHeader};
	const char* hdr_name[] = {"voila_device.cuh"};
	if (nvrtcCreateProgram(&prog, source.c_str(), "voila_pipelines.cu", 1, hdr_src, hdr_name) != NVRTC_SUCCESS) {
		throw Error(5, "nvrtcCreateProgram failed");
	}
	nvrtcResult rc = nvrtcCompileProgram(prog, kNumOpts, kOpts);
	size_t log_size = 0;
	nvrtcGetProgramLogSize(prog, &log_size);
	std::string log(log_size, '\0');
	if (log_size > 1) {
		nvrtcGetProgramLog(prog, &log[0]);
	}
	if (log_out) {
		*log_out = log;
	}
	if (rc != NVRTC_SUCCESS) {
		nvrtcDestroyProgram(&prog);
		throw Error(5, std::string("NVRTC: ") + nvrtcGetErrorString(rc) + "\n" + log);
	}
	size_t n = 0;
	nvrtcGetCUBINSize(prog, &n);
	std::string bin(n, '\0');
	nvrtcGetCUBIN(prog, &bin[0]);
	nvrtcDestroyProgram(&prog);

	mkdirs(dir);
	const std::string tmp = path + ".tmp" + std::to_string(getpid());
	{
		std::ofstream out(tmp, std::ios::binary);
		out.write(bin.data(), (std::streamsize)bin.size());
	}
	std::rename(tmp.c_str(), path.c_str());
	return bin;
}

std::shared_ptr<JitModule> jit_compile(const std::string& source, std::string* log_out)
{
	static std::mutex mu;
	static std::map<std::string, std::weak_ptr<JitModule>> loaded;
	const std::string key = key_of(source);
	{
		std::lock_guard<std::mutex> g(mu);
		auto it = loaded.find(key);
		if (it != loaded.end()) {
			if (auto m = it->second.lock()) {
				return m;
			}
		}
	}
	std::string bin = jit_cubin(source, log_out);
	auto mod = std::shared_ptr<JitModule>(new JitModule(), [](JitModule* m) {
		if (m->lib) {
			cudaLibraryUnload(m->lib);
		}
		delete m;
	});
	VC_CHECK_CUDA(cudaLibraryLoadData(&mod->lib, bin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
	std::lock_guard<std::mutex> g(mu);
	loaded[key] = mod;
	return mod;
}

} // namespace vc
