"""usap-b200: B200-native stochastic block partitioning (uSAP's SBP path).

Public API (all GPU work goes through the C ABI in include/usap.h):

* ``Graph_P``     the reference's class shape: params, partition(),
                  get_partitions(), num_nodes(), num_edges()
* ``partition``   one-shot solve from edge arrays
* ``batch_partition``  many graphs x chains at once on one GPU
* ``evaluate``    bf::evaluate's scores, returned as a dict
* ``Context``     a graph resident in HBM, plus phase-level replay ops
* ``Server``      a partition service: submit requests, collect by ticket
* ``generator``   seeded DC-SBM graphs
"""
from . import generator  # noqa: F401

__all__ = ["Graph_P", "Context", "Server", "partition", "batch_partition", "evaluate", "generator"]


def __getattr__(name):
    if name in ("Graph_P", "Context", "Server", "partition", "batch_partition", "evaluate"):
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
