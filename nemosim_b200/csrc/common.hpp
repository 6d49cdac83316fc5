// common.hpp -- error type, status codes and neuron-type descriptors shared
// by the host side of the B200 backend.
#pragma once

#include <stdint.h>

#include <stdexcept>
#include <string>

#include "../../include/nemo_b200.h"

namespace nemo_b200 {

// nemo::exception (src/nemo/exception.hpp:23): a message with a status code
class Error : public std::runtime_error {
public:
	Error(int code, const std::string& msg) : std::runtime_error(msg), m_code(code) {}
	int code() const { return m_code; }
private:
	int m_code;
};

std::string format(const char* fmt, ...) __attribute__((format(printf, 1, 2)));

#define NB_THROW(code, ...) throw ::nemo_b200::Error((code), ::nemo_b200::format(__VA_ARGS__))

// A neuron type as its .ini descriptor describes it
// (src/nemo/NeuronType.cpp:91-156), bound to the kernel of this backend
// that updates it (src/nemo/cuda/Neurons.cpp:43 binds the CUDA plugin of
// the type instead).  KIND_NONE: the backend has no kernel for the type.
enum NeuronKind {
	KIND_NONE = -1,
	KIND_IZHIKEVICH = 0,
	KIND_IF_CURR_EXP = 1,
	KIND_POISSON = 2,
	KIND_INPUT = 3,
	KIND_IZHIKEVICH_RS = 4,
	KIND_KURAMOTO = 5,
	KIND_COUNT = 6
};

struct NeuronTypeDesc {
	std::string name;
	NeuronKind kind = KIND_NONE;
	unsigned nparam = 0;
	unsigned nstate = 0;
	unsigned mpot = 0;        // state index of the membrane potential
	bool nrand = false;       // uses the normal RNG
	unsigned history = 1;     // state history length
	bool rcmSources = false, rcmDelays = false, rcmForward = false, rcmWeights = false;
	bool cpu = false, cuda = false;  // [backends]
	std::string pluginDir;    // directory of the .ini file
};

// The kernels compiled into the step loop, by kind: the name of the type
// each implements and the parameter, state and RNG layout it expects
// (src/nemo/plugins/Izhikevich.h, IF_curr_exp.h; the .ini descriptors).
struct KernelLayout {
	const char* name;
	unsigned nparam, nstate;
	bool nrand;
	unsigned history;  // state history the kernel keeps
};
extern const KernelLayout KERNELS[KIND_COUNT];
// Q(31-f).f with f = 20 (src/nemo/ConfigurationImpl.cpp:22)
constexpr unsigned FRACTIONAL_BITS = 20;
// longest firing history / STDP window (src/nemo/StdpFunction.cpp:151)
constexpr unsigned MAX_HISTORY = 64;
// neuron ids are packed with 6 delay bits into 32-bit words on the device
constexpr unsigned MAX_NEURONS = 1u << 26;

// fx_toFix of src/nemo/fixedpoint.cpp:17-28 (throws a plain runtime error,
// which the C API reports as NEMO_UNKNOWN_ERROR as the reference does)
int32_t fx_toFix(float f);
inline float fx_toFloat(int32_t v) { return (float) v / (float) (1 << FRACTIONAL_BITS); }

} // namespace nemo_b200
