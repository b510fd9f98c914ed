"""Generated neuron models (placeholder until the generator lands)."""
from .lowering import ModelUnsupported


def lower_model(script, g, model, res, thr, rst, refractory, method, dtype, ops):
    raise ModelUnsupported(f"{g.name}: the model is neither the LIF nor the COBAHH system")
