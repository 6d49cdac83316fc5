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

// The compiled-in neuron types.  Parameter/state counts, membrane-potential
// index and RNG use follow the .ini descriptors
// (src/nemo/plugins/{Izhikevich,IF_curr_exp,PoissonSource,Input}.ini) and
// the index headers (src/nemo/plugins/Izhikevich.h, IF_curr_exp.h).
enum NeuronKind { KIND_IZHIKEVICH = 0, KIND_IF_CURR_EXP = 1, KIND_POISSON = 2, KIND_INPUT = 3 };

struct NeuronTypeDesc {
	const char* name;
	NeuronKind kind;
	unsigned nparam;
	unsigned nstate;
	unsigned mpot;     // state index of the membrane potential
};

extern const NeuronTypeDesc NEURON_TYPES[4];
const NeuronTypeDesc* find_neuron_type(const std::string& name);

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
