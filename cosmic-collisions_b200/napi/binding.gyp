{
  "targets": [{
    "target_name": "ccstep",
    "sources": ["ccstep_napi.c"],
    "include_dirs": ["../../include"],
    "libraries": ["-L<(module_root_dir)/..", "-lccstep", "-Wl,-rpath,<(module_root_dir)/.."],
    "cflags": ["-std=c11", "-O2"]
  }]
}
