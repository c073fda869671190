// path tracer restatement (filled in later)
