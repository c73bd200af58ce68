"""``POST /solve`` in front of the device request loop.

The wire format is the reference server's (crates/mr-server/src/lib.rs:147-171):
the body is ``{"simple_route_json": {...}, "problem_soup": ..., "resolution":
...}`` (``problem_soup`` accepted and ignored, ``resolution`` an optional cell
size), a success is ``200 {"solution_soup": [pcb_trace, ...]}`` and a failure
``{"error": "..."}`` with 400 for a malformed body or an invalid endpoint /
grid and 500 for a backend failure (router_error_response, :455-469).

Each request is rasterised on the handler's thread (``srj.rasterize`` at the
server's resolution policy, ``choose_resolution``), submitted to one shared
``mrc_server`` and answered when its result is on the host.  Handlers run on
their own threads (ThreadingHTTPServer), so requests that arrive while others
are on the GPU are admitted by the server's HBM budget and merged into shared
launches: continuous batching behind the reference's ``/solve`` seam.

What a request is answered with: the canonical isolated ("alone") path of
every connection, the path NegotiatedRouter's provider batch computes
(negotiated.rs:1386-1454), window first then whole board.  The reference's
handler continues from those paths through negotiation rounds and the CPU
legalisation pass, which this engine does not run behind this seam.

  python -m mrcuda.solve_http --port 8080     (from metal-route_b200/)
"""
from __future__ import annotations

import argparse
import json
import threading
from http.server import BaseHTTPRequestHandler, ThreadingHTTPServer
from typing import Optional, Tuple

from . import api
from .srj import choose_resolution, rasterize, solution_soup


class SolveService:
    """The handler logic, independent of HTTP: one engine, one request loop."""

    def __init__(self, engine: "api.Engine", slots: int = 2, hbm_fraction: float = 0.8, solve_layers: int = 1,
                 clearance_cells: int = 0):
        self.engine = engine
        self.server = engine.server(slots=slots, hbm_fraction=hbm_fraction)
        self.solve_layers = solve_layers
        self.clearance_cells = clearance_cells

    def solve(self, body) -> Tuple[int, dict]:
        if not isinstance(body, dict) or not isinstance(body.get("simple_route_json"), dict):
            return 400, {"error": "invalid request body: missing field `simple_route_json`"}
        srj = body["simple_route_json"]
        try:
            if "bounds" not in srj or "layerCount" not in srj:
                raise KeyError("bounds" if "bounds" not in srj else "layerCount")
            res = body.get("resolution")
            resolution = choose_resolution(srj, None if res is None else float(res))
            prob = rasterize(srj, resolution, layers=self.solve_layers, clearance_cells=self.clearance_cells)
        except (KeyError, TypeError, ValueError) as e:
            return 400, {"error": f"invalid request body: {e}"}
        try:
            result, _ = self.server.wait(self.server.submit(prob.request, retry_full=True))
        except (api.InvalidEndpoint, api.MalformedGrid, api.InvalidArgument) as e:
            return 400, {"error": str(e)}
        except api.RouterError as e:
            return 500, {"error": f"backend unavailable: {e}"}
        return 200, {"solution_soup": solution_soup(prob, result.paths)}

    def close(self):
        self.server.close()


def make_handler(service: SolveService):
    class Handler(BaseHTTPRequestHandler):
        protocol_version = "HTTP/1.1"

        def _reply(self, status: int, obj: dict):
            data = json.dumps(obj).encode()
            self.send_response(status)
            self.send_header("Content-Type", "application/json")
            self.send_header("Content-Length", str(len(data)))
            self.end_headers()
            self.wfile.write(data)

        def do_POST(self):  # noqa: N802 (http.server naming)
            if self.path.rstrip("/") != "/solve":
                self._reply(404, {"error": "not found"})
                return
            n = int(self.headers.get("Content-Length", "0") or 0)
            try:
                body = json.loads(self.rfile.read(n) or b"null")
            except ValueError as e:
                self._reply(400, {"error": f"invalid request body: {e}"})
                return
            status, obj = service.solve(body)
            self._reply(status, obj)

        def log_message(self, fmt, *args):  # quiet
            pass

    return Handler


def serve(service: SolveService, host: str = "127.0.0.1", port: int = 8080,
          ready: Optional[threading.Event] = None) -> ThreadingHTTPServer:
    """Start the HTTP server on a daemon thread; returns it (``.shutdown()`` stops it)."""
    httpd = ThreadingHTTPServer((host, port), make_handler(service))
    httpd.daemon_threads = True
    t = threading.Thread(target=httpd.serve_forever, daemon=True)
    t.start()
    if ready is not None:
        ready.set()
    return httpd


def main():
    ap = argparse.ArgumentParser(description="POST /solve over the CUDA request loop")
    ap.add_argument("--host", default="127.0.0.1")
    ap.add_argument("--port", type=int, default=8080)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--slots", type=int, default=2)
    ap.add_argument("--solve-layers", type=int, default=1)
    args = ap.parse_args()
    eng = api.Engine(args.device)
    svc = SolveService(eng, slots=args.slots, solve_layers=args.solve_layers)
    httpd = serve(svc, args.host, args.port)
    try:
        threading.Event().wait()
    except KeyboardInterrupt:
        pass
    httpd.shutdown()
    svc.close()
    eng.close()


if __name__ == "__main__":
    main()
