// plugins.cpp -- neuron types from their .ini descriptors.
//
// A type is described by <name>.ini (src/nemo/NeuronType.cpp:91-156), found
// in the directories added with nemo_add_plugin_path, then in the user's
// plugin directory ~/.nemo/plugins, then in the library's own plugin
// directory (src/nemo/NeuronType.cpp:45-70).  The library's directory is
// plugins/ beside the directory that holds libnemo_b200.so (the reference
// installs its descriptors under <libdir>/nemo/plugins).  Where the
// reference then loads <plugin dir>/cuda/lib<name>.so for the update
// (src/nemo/cuda/Neurons.cpp:43), this backend binds the type by name to a
// kernel compiled into its step loop, whose layout the descriptor must
// match (checked when a simulation is created).
#include "plugins.hpp"

#include <ctype.h>
#include <dlfcn.h>
#include <errno.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <fstream>
#include <map>
#include <mutex>
#include <set>

namespace nemo_b200 {

// the kernels of kernels.cuh, by kind
const KernelLayout KERNELS[KIND_COUNT] = {
	{ "Izhikevich", 5, 2, true, 1 },
	{ "IF_curr_exp", 9, 4, false, 1 },
	{ "PoissonSource", 1, 0, true, 1 },
	{ "Input", 0, 0, false, 1 },
	{ "IzhikevichRS", 0, 2, false, 1 },
	{ "Kuramoto", 1, 1, false, 32 },
};

namespace {

std::mutex g_pathLock;
std::set<std::string> g_extraPaths;  // ordered, as the reference's std::set of paths

bool exists(const std::string& p)
{
	struct stat st;
	return stat(p.c_str(), &st) == 0;
}

std::string trim(const std::string& s)
{
	size_t b = 0, e = s.size();
	while(b < e && isspace((unsigned char) s[b])) ++b;
	while(e > b && isspace((unsigned char) s[e - 1])) --e;
	return s.substr(b, e - b);
}

// unsigned as the reference's lexical_cast accepts it (decimal digits)
bool parseUnsigned(const std::string& v, unsigned* out)
{
	if(v.empty() || v.size() > 9) return false;
	unsigned x = 0;
	for(char c : v) {
		if(c < '0' || c > '9') return false;
		x = x * 10 + (unsigned) (c - '0');
	}
	*out = x;
	return true;
}

// bool as boost::program_options accepts it
bool parseBool(const std::string& v, bool* out)
{
	std::string s;
	for(char c : v) s.push_back((char) tolower((unsigned char) c));
	if(s.empty() || s == "on" || s == "yes" || s == "1" || s == "true") {
		*out = true;
		return true;
	}
	if(s == "off" || s == "no" || s == "0" || s == "false") {
		*out = false;
		return true;
	}
	return false;
}

} // namespace

void addPluginPath(const std::string& dir)
{
	// Plugin::addPath (src/nemo/Plugin.cpp:185-195)
	if(!exists(dir)) NB_THROW(NEMO_DL_ERROR, "User-specified path %s could not be found", dir.c_str());
	std::lock_guard<std::mutex> lock(g_pathLock);
	g_extraPaths.insert(dir);
}

std::string systemPluginDirectory()
{
	Dl_info info;
	if(dladdr((void*) &systemPluginDirectory, &info) && info.dli_fname) {
		std::string lib(info.dli_fname);
		const size_t slash = lib.rfind('/');
		const std::string libdir = slash == std::string::npos ? std::string(".") : lib.substr(0, slash);
		return libdir + "/../plugins";
	}
	return "plugins";
}

// configurationFile (src/nemo/NeuronType.cpp:45-70)
std::string pluginConfigurationFile(const std::string& name)
{
	{
		std::lock_guard<std::mutex> lock(g_pathLock);
		for(const std::string& dir : g_extraPaths) {
			const std::string p = dir + "/" + name + ".ini";
			if(exists(p)) return p;
		}
	}
	const char* home = getenv("HOME");
	if(!home) NB_THROW(NEMO_DL_ERROR, "Could not locate user's home directory when searching for plugins");
	const std::string user = std::string(home) + "/.nemo/plugins/" + name + ".ini";
	if(exists(user)) return user;
	const std::string sys = systemPluginDirectory();
	if(!exists(sys)) NB_THROW(NEMO_DL_ERROR, "System plugin path does not exist: %s", sys.c_str());
	const std::string p = sys + "/" + name + ".ini";
	if(exists(p)) return p;
	NB_THROW(NEMO_INVALID_INPUT, "Could not find .ini file for plugin %s", name.c_str());
}

// NeuronType::parseConfigurationFile (src/nemo/NeuronType.cpp:91-156): the
// keys of a boost::program_options configuration file -- "key=value"
// lines, "[section]" headers prefixing the keys that follow with
// "section.", '#' starting a comment -- with four required keys and the
// others defaulted; an unknown key, a repeated key, a line without '=' or a
// value of the wrong type is a parse error.
NeuronTypeDesc parseNeuronType(const std::string& name)
{
	const std::string file = pluginConfigurationFile(name);
	std::ifstream in(file);
	if(!in.is_open()) {
		NB_THROW(NEMO_IO_ERROR, "Failed to open neuron model configuration file %s: %s", file.c_str(), strerror(errno));
	}
	enum Kind { UNSIGNED, BOOL };
	const std::map<std::string, Kind> known = {
		{ "parameters", UNSIGNED }, { "state-variables", UNSIGNED }, { "membrane-potential", UNSIGNED },
		{ "history", UNSIGNED }, { "rng.normal", BOOL }, { "rcm.sources", BOOL }, { "rcm.delays", BOOL },
		{ "rcm.forward", BOOL }, { "rcm.weights", BOOL }, { "backends.cpu", BOOL }, { "backends.cuda", BOOL },
	};
	std::map<std::string, std::string> values;
	std::string section, line;
	auto fail = [&](const std::string& why) {
		NB_THROW(NEMO_INVALID_INPUT, "Error parsing neuron model configuration file %s: %s", file.c_str(),
				why.c_str());
	};
	while(std::getline(in, line)) {
		const size_t hash = line.find('#');
		if(hash != std::string::npos) line.erase(hash);
		line = trim(line);
		if(line.empty()) continue;
		if(line.front() == '[') {
			if(line.back() != ']') fail("invalid section header '" + line + "'");
			section = trim(line.substr(1, line.size() - 2)) + ".";
			continue;
		}
		const size_t eq = line.find('=');
		if(eq == std::string::npos) fail("invalid line '" + line + "'");
		const std::string key = section + trim(line.substr(0, eq));
		const std::string value = trim(line.substr(eq + 1));
		const auto k = known.find(key);
		if(k == known.end()) fail("unrecognised option '" + key + "'");
		if(values.count(key)) fail("option '" + key + "' cannot be specified more than once");
		if(k->second == UNSIGNED) {
			unsigned x;
			if(!parseUnsigned(value, &x)) fail("the argument ('" + value + "') for option '" + key + "' is invalid");
		} else {
			bool b;
			if(!parseBool(value, &b)) fail("the argument ('" + value + "') for option '" + key + "' is invalid");
		}
		values[key] = value;
	}
	auto required = [&](const char* key) -> const std::string& {
		auto it = values.find(key);
		if(it == values.end()) {
			NB_THROW(NEMO_INVALID_INPUT, "Missing parameter '%s' in configuration file %s", key, file.c_str());
		}
		return it->second;
	};
	auto flag = [&](const char* key, bool dflt) {
		auto it = values.find(key);
		bool b = dflt;
		if(it != values.end()) parseBool(it->second, &b);
		return b;
	};
	NeuronTypeDesc d;
	d.name = name;
	parseUnsigned(required("parameters"), &d.nparam);
	parseUnsigned(required("state-variables"), &d.nstate);
	parseUnsigned(required("membrane-potential"), &d.mpot);
	parseBool(required("rng.normal"), &d.nrand);
	d.rcmSources = flag("rcm.sources", false);
	d.rcmDelays = flag("rcm.delays", false);
	d.rcmForward = flag("rcm.forward", false);
	d.rcmWeights = flag("rcm.weights", false);
	d.history = 1;
	if(values.count("history")) parseUnsigned(values["history"], &d.history);
	d.cpu = flag("backends.cpu", false);
	d.cuda = flag("backends.cuda", false);
	const size_t slash = file.rfind('/');
	d.pluginDir = slash == std::string::npos ? std::string(".") : file.substr(0, slash);
	d.kind = KIND_NONE;
	for(int k = 0; k < KIND_COUNT; ++k) {
		if(name == KERNELS[k].name) d.kind = (NeuronKind) k;
	}
	return d;
}

void checkKernelBinding(const NeuronTypeDesc& d)
{
	if(d.kind == KIND_NONE) {
		NB_THROW(NEMO_DL_ERROR, "Error when loading plugin %s: the B200 backend has no kernel for neuron type %s",
				d.name.c_str(), d.name.c_str());
	}
	const KernelLayout& k = KERNELS[d.kind];
	if(d.nparam != k.nparam || d.nstate != k.nstate || d.nrand != k.nrand || d.history != k.history) {
		NB_THROW(NEMO_DL_ERROR,
				"Error when loading plugin %s: the descriptor in %s gives %u parameters, %u state variables, "
				"normal RNG %s and history %u; the B200 kernel for %s expects %u, %u, %s and %u",
				d.name.c_str(), d.pluginDir.c_str(), d.nparam, d.nstate, d.nrand ? "on" : "off", d.history, k.name,
				k.nparam, k.nstate, k.nrand ? "on" : "off", k.history);
	}
	if(d.mpot >= d.nstate && d.nstate > 0) {
		NB_THROW(NEMO_DL_ERROR, "Error when loading plugin %s: membrane-potential index %u is not a state variable",
				d.name.c_str(), d.mpot);
	}
}

} // namespace nemo_b200
