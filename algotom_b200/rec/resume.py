"""Resumable slab streaming: a host-side manifest of finished slabs.

algotom has no checkpointing on this path; its example scripts restart a
long reconstruction by slice range (``--start`` / ``--stop``,
``examples/common_data_processing_workflow/full_reconstruction_cli.py:38-41``).
Here ``fbp_reconstruction(..., out=<persistent array>, resume=<path>)``
streams a host stack through the device slab by slab and records in a JSON
manifest every slab whose reconstruction has reached ``out``; run again
after an interruption with the same arguments, it skips those slabs.

The manifest names the stack shape and the parameters that define the
result, so a manifest written for other data or settings is refused
instead of being resumed.  It is rewritten atomically (temporary file,
then rename), so an interruption while it is written leaves the previous
version.
"""
import json
import os


class SlabManifest:
    """Finished slabs ``(first slice, count)`` of one streamed reconstruction.

    ``key`` is a JSON-serialisable description of the job (shape, centre,
    angles digest, filter settings, slab size); :meth:`open` refuses a file
    whose key differs.
    """

    VERSION = 1

    def __init__(self, path, key, done=None):
        self.path = path
        self.key = key
        self.done = set(done or ())

    @classmethod
    def open(cls, path, key):
        """Load the manifest at ``path`` (or start an empty one if there is
        none).  Raises ValueError if it belongs to another job."""
        if not os.path.exists(path):
            return cls(path, key)
        with open(path) as f:
            try:
                d = json.load(f)
            except ValueError as e:
                raise ValueError("resume manifest %s is unreadable: %s"
                                 % (path, e))
        if d.get("version") != cls.VERSION or d.get("key") != key:
            raise ValueError("resume manifest %s belongs to another "
                             "reconstruction (shape, centre, angles or "
                             "settings differ); remove it to start over"
                             % path)
        return cls(path, key, (tuple(s) for s in d.get("done", ())))

    def is_done(self, span):
        return tuple(span) in self.done

    def mark(self, spans):
        """Record finished slabs and rewrite the file."""
        new = set(tuple(s) for s in spans) - self.done
        if not new:
            return
        self.done |= new
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump({"version": self.VERSION, "key": self.key,
                       "done": sorted(self.done)}, f)
        os.replace(tmp, self.path)
