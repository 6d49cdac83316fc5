/* Stand-in for src/nemo/types.hpp: a synapse as the generator yields it. */
#ifndef NEMO_TYPES_HPP
#define NEMO_TYPES_HPP
#include <stddef.h>
#include <nemo/config.h>
#include "internal_types.h"
#include "Neuron.hpp"
namespace nemo {
struct AxonTerminal
{
	id32_t id;
	nidx_t target;
	float weight;
	bool plastic;
	AxonTerminal() : id(~0), target(~0), weight(0.0f), plastic(false) { }
	AxonTerminal(id32_t id, nidx_t t, float w, bool p) : id(id), target(t), weight(w), plastic(p) { }
};
class Synapse
{
	public :
		Synapse() : source(0), delay(0) {}
		Synapse(nidx_t source, delay_t delay, const AxonTerminal& terminal) :
			source(source), delay(delay), terminal(terminal) { }
		nidx_t source;
		delay_t delay;
		AxonTerminal terminal;
		id32_t id() const { return terminal.id; }
		nidx_t target() const { return terminal.target; }
		unsigned char plastic() const { return terminal.plastic; }
		float weight() const { return terminal.weight; }
};
}
#endif
