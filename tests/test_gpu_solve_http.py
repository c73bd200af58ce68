"""POST /solve over HTTP in front of the device request loop.

Generated SimpleRouteJson problems (the reference bench's generator) are posted
one at a time and then all at once from several threads; the answers must be
identical either way (the concurrent ones share launches in the request loop)
and equal the solution soup of the oracle's paths on the same rasterised
request.  Malformed bodies get the reference's 400 + {"error"} reply.
"""
import json
import urllib.error
import urllib.request
from concurrent.futures import ThreadPoolExecutor

import pytest

import mrcuda
from mrcuda import srj
from mrcuda.solve_http import SolveService, serve

pytestmark = pytest.mark.gpu


def _post(port, body: bytes):
    req = urllib.request.Request(f"http://127.0.0.1:{port}/solve", data=body,
                                 headers={"Content-Type": "application/json"}, method="POST")
    try:
        with urllib.request.urlopen(req, timeout=120) as r:
            return r.status, json.loads(r.read())
    except urllib.error.HTTPError as e:
        return e.code, json.loads(e.read())


def test_solve_over_http(oracle):
    eng = mrcuda.Engine(0)
    svc = SolveService(eng, slots=2, solve_layers=2)
    httpd = serve(svc, "127.0.0.1", 0)
    port = httpd.server_address[1]
    try:
        problems = [srj.generate_problem(seed, 30.0, 8, 24) for seed in range(1, 9)]
        bodies = [json.dumps({"simple_route_json": p, "resolution": 0.25, "problem_soup": None}).encode()
                  for p in problems]
        one_by_one = [_post(port, b) for b in bodies]
        with ThreadPoolExecutor(len(bodies)) as ex:
            together = list(ex.map(lambda b: _post(port, b), bodies))
        assert together == one_by_one
        for p, (status, body) in zip(problems, one_by_one):
            assert status == 200, body
            prob = srj.rasterize(p, 0.25, layers=2)
            paths, _ = oracle.isolated_batch(prob.request, retry_full=True, mode="astar")
            assert body["solution_soup"] == srj.solution_soup(prob, paths)
            assert len(body["solution_soup"]) >= 1
        st = svc.server.stats()
        assert st["completed"] == 2 * len(bodies) and st["failed"] == 0
        # the reference's error replies
        assert _post(port, b"{not json")[0] == 400
        status, body = _post(port, json.dumps({"resolution": 0.5}).encode())
        assert status == 400 and "simple_route_json" in body["error"]
        status, body = _post(port, json.dumps({"simple_route_json": {"connections": []}}).encode())
        assert status == 400 and "error" in body
    finally:
        httpd.shutdown()
        svc.close()
        eng.close()
