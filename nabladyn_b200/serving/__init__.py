"""Serving many independent MD replicas on one GPU: continuous batching into persistent kernels.

``ReplicaServer`` keeps replicas resident in one device pool, admits requests as slots and HBM
budget free up, advances every active replica by a per-replica budget of NVT steps in one
launch of the replica kernel (nd_serve_run: one CTA per replica, whole steps inside the CTA),
and hands back each finished replica's frame with its latency.
"""

from ._server import ReplicaRequest, ReplicaResult, ReplicaServer
from ._workload import serving_requests

__all__ = ("ReplicaRequest", "ReplicaResult", "ReplicaServer", "serving_requests")
